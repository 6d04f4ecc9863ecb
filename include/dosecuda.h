/*
 * dosecuda.h — C ABI of the B200 (sm_100a) DoseCUDA dose engines.
 *
 * This is the drop-in boundary for the reference's `dose_kernels` CPython
 * extension (DoseCUDA/dose_kernels/dosemodule.cu).  Each host entry point
 * below replaces one function of that module's method table
 * (dosemodule.cu:560-580) and keeps its argument meaning, its output, and its
 * error classes; the Python shim `dosecuda_b200/dose_kernels.py` maps the
 * reference's duck-typed (model, volume, beam, gpu_id) objects onto these
 * plain-pointer calls.
 *
 * Conventions
 *  - Volumes are C-contiguous float32 arrays of shape (nz, ny, nx), index
 *    i + nx*(j + ny*k)  (reference CudaClasses.cuh:96-98).
 *  - spacing/origin/iso are in mm, in (x, y, z) order.  The engines accept
 *    three spacings; the reference itself only reads spacing[0]
 *    (dosemodule.cu:146,300,471), and the `dose_kernels` shim passes
 *    spacing[0] three times to reproduce that.
 *  - Angles are in degrees, as the caller gives them; the +180 degree gantry
 *    offset of the reference (dosemodule.cu:152,304,477) is applied inside.
 *    The gantry angle is a double because the reference forms
 *    fmodf(gantry + 180, 360) from the Python float before rounding.
 *  - Every function returns DC_OK (0) or an error code; dc_last_error()
 *    returns the message of the calling thread's last failure.
 *  - Host entry points (no suffix) take host pointers and are synchronous,
 *    like the reference.  The *_dev entry points take device pointers and a
 *    cudaStream_t (passed as void*; NULL = legacy default stream), enqueue
 *    the work and return without synchronising.
 *  - Outputs are caller-owned buffers of nz*ny*nx floats.
 */
#ifndef DOSECUDA_H
#define DOSECUDA_H

#ifdef __cplusplus
extern "C" {
#endif

#define DC_OK 0
#define DC_ERR_VALUE 1   /* bad argument: the reference raises ValueError    */
#define DC_ERR_MEMORY 2  /* host allocation failed: MemoryError            */
#define DC_ERR_CUDA 3    /* CUDA runtime/launch failure: RuntimeError       */

/* Photon beam model: the scalar and 1-D array attributes that the reference
 * reads from an IMRTPhotonEnergy object (dosemodule.cu:400-437).  The CCCS
 * kernel table is passed as its six logical columns (kernel.csv: theta in
 * degrees, Am, am, Bm, bm, ray_length in cm), n_cones rows each; the
 * reference reads the same numbers column-major from the pandas-built array
 * (IMRTClasses.cu:292-297). */
typedef struct dc_photon_model {
    int n_profile_points;
    const float *profile_radius;        /* mm, ascending            */
    const float *profile_intensities;
    const float *profile_softening;
    int n_spectral_energies;
    const float *spectrum_attenuation_coefficients;  /* 1/cm */
    const float *spectrum_primary_weights;
    const float *spectrum_scatter_weights;
    float mu_calibration;
    float primary_source_distance;      /* mm */
    float scatter_source_distance;      /* mm */
    float primary_source_size;          /* mm */
    float scatter_source_size;          /* mm */
    float mlc_distance;                 /* mm */
    float scatter_source_weight;
    float electron_attenuation;
    float electron_source_weight;
    float electron_fitted_dmax;
    float jaw_transmission;             /* parsed, unused (as the reference) */
    float mlc_transmission;             /* parsed, unused (as the reference) */
    int has_xjaws;                      /* parsed, unused (as the reference) */
    int has_yjaws;                      /* parsed, unused (as the reference) */
    int n_cones;                        /* rows of the kernel table (6)      */
    const float *kernel_theta_deg;
    const float *kernel_Am;
    const float *kernel_am;
    const float *kernel_Bm;
    const float *kernel_bm;
    const float *kernel_ray_length;     /* cm */
} dc_photon_model;

/* One photon control point (reference IMRTControlPoint, plan_imrt.py:95-105).
 * MLC leaf pairs are passed as four logical columns of n_mlc_pairs values:
 * x1, x2 (leaf tips, mm at isocentre), y_offset and y_width (mm); the
 * reference reads them the same way (dosemodule.cu:228-240). */
typedef struct dc_control_point {
    float iso[3];
    float mu;
    double gantry_deg;  /* double: the reference adds 180 in double before
                           rounding to float (dosemodule.cu:477) */
    float collimator_deg;
    float couch_deg;
    int n_mlc_pairs;
    const float *mlc_x1;
    const float *mlc_x2;
    const float *mlc_y_offset;
    const float *mlc_y_width;
} dc_control_point;

/* ------------------------------------------------------------------ */
/* Library                                                             */
/* ------------------------------------------------------------------ */

/* Message of the calling thread's last failed call ("" if none). */
const char *dc_last_error(void);

/* Whether the host buffer [host, host + bytes) is page-locked memory mapped
 * into gpu_id's address space as one allocation (cudaHostAlloc /
 * cudaHostRegister, e.g. torch's pinned allocator).  The host-buffer entry
 * points (dc_proton_raytrace, dc_proton_spot, dc_photon_dose) let their
 * kernels read the input WET and write the result in place in such buffers,
 * so the transfers overlap the kernels instead of following them; other
 * buffers are copied.  No reference counterpart. */
int dc_host_buffer_mapped(int gpu_id, const void *host, unsigned long long bytes, int *mapped);

/* Debug-build bounds report (no reference counterpart).  A library built
 * with -DDC_DEBUG_BOUNDS checks the index of every instrumented global
 * access of the dose kernels against its buffer; the first violation is
 * recorded (site << 48 | index) and the access skipped.  This call waits for
 * the device, returns *enabled = 1 for such a build (0 otherwise) and the
 * first recorded violation since the last call (0: none), and clears it. */
int dc_debug_bounds(int gpu_id, unsigned long long *violation, int *enabled);

/* ---- Linear dose basis (segment weights of a photon beam) -------------
 * No reference counterpart: the reference's plan loop (plan_imrt.py:140-156)
 * computes each control point's dose and adds it times its output factor.
 * With those doses kept on the device as basis[b][v] (n_basis volumes of
 * n_vox floats), the plan dose for any segment weights and its adjoint are:
 *
 * dc_basis_combine_dev: out[v] = running acc over b (in order) of
 *   acc = float32(double(acc) + double(basis[b][v]) * coef[b]), starting
 *   from out[v]: the plan loop's arithmetic, so coef = output factors gives
 *   its result bit for bit.  coef_dev: n_basis doubles on the device.
 * dc_basis_adjoint_dev: grad_out[b] = sum_v grad_dose[v] * basis[b][v] in
 *   float64 (grad_out_dev: n_basis doubles, overwritten).
 * Both are asynchronous on `stream` and allocate nothing. */
int dc_basis_combine_dev(int gpu_id, const float *basis, int n_basis, long long n_vox, const double *coef_dev,
                         float *out_dev, void *stream);
int dc_basis_adjoint_dev(int gpu_id, const float *basis, int n_basis, long long n_vox, const float *grad_dose_dev,
                         double *grad_out_dev, void *stream);

/* ABI version (major*10000 + minor*100 + patch). */
int dc_version(void);

/* Number of CUDA devices visible (0 when none), or -1 on a driver error. */
int dc_device_count(void);

/* Free the cached device buffers, textures and streams held for gpu_id. */
int dc_release_device(int gpu_id);

/* No counterpart in the reference (its ray trace, CudaClasses.cu:180-228,
 * is the only mode).  How photon calls on gpu_id compute the radiological
 * depth that TERMA attenuates with:
 *   DC_DEPTH_MARCH   (0): the reference's per-voxel 1 mm march, sample
 *                         for sample;
 *   DC_DEPTH_LATTICE (1): the default: the density integrated once along a
 *                         beam's-eye-view lattice of rays from the source and
 *                         interpolated per voxel, with the reference's exact
 *                         sample count, its boundary samples fetched exactly,
 *                         and the exact march wherever neighbouring lattice
 *                         rays disagree by more than 0.03 cm of WET (weighed
 *                         by the voxel's density, up to water's) without a
 *                         near-linear variation between them, and for
 *                         shallow voxels (electron contamination range)
 *                         wherever they disagree by more than 0.001 cm.  An
 *                         approximation: TERMA typically within 0.15 % of
 *                         the march, up to ~1 % on rays grazing a voxelised
 *                         body surface; the dose within 0.1 % of Dmax on the
 *                         tested geometries.
 * Applies to calls enqueued after it returns; proton WET always uses the
 * march. */
#define DC_DEPTH_MARCH 0
#define DC_DEPTH_LATTICE 1
int dc_photon_set_depth_mode(int gpu_id, int mode);
int dc_photon_get_depth_mode(int gpu_id, int *mode);
/* Voxels the last lattice depth pass of a photon call on gpu_id marched
 * exactly (its fallback); -1 when the last pass marched every voxel or none
 * ran.  Synchronises the device. */
int dc_photon_depth_stats(int gpu_id, long long *marched);
/* Self-test of the head transmission's leaf-pair skip (replaces nothing in
 * the reference, which evaluates every pair, headTransmission
 * IMRTClasses.cu:120-150): *largest_unsaturated = the largest float x in
 * [3, 4.5] for which the device's erff(x) != 1 or erff(-x) != -1 (0 if
 * none), *skip_bound = the edge argument beyond which the kernel skips a
 * pair.  The skip leaves every sum bitwise unchanged when
 * largest_unsaturated <= skip_bound.  Synchronous. */
int dc_photon_head_selftest(int gpu_id, float *largest_unsaturated, float *skip_bound);

/* Kernel timing: when enabled, every kernel the library launches is
 * bracketed by CUDA events on its own stream.  dc_profile_read synchronises
 * the device and returns, per kernel name, the launch count and the summed
 * device time (ms).  Returns the number of kernels written (<= max). */
int dc_profile_enable(int gpu_id, int on);
int dc_profile_reset(int gpu_id);
int dc_profile_read(int gpu_id, int max, const char **names, int *launches, double *total_ms);

/* Measures the rate of trilinear float2 3D texture fetches the device
 * delivers in the CCCS kernel's access pattern (all SMs, full occupancy):
 * the roof of the texture-bound ray-march kernels.  Synchronous, ~1 ms.
 * No counterpart in the reference. */
int dc_texture_fetch_rate(int gpu_id, double *fetches_per_s);

/* ------------------------------------------------------------------ */
/* Proton: water-equivalent thickness (WET) ray trace + BEV smoothing   */
/* Replaces dose_kernels.proton_raytrace_cuda                           */
/* (dosemodule.cu:104-201 -> IMPTClasses.cu:274-299).                   */
/* Output: smoothed WET in cm.                                          */
/* ------------------------------------------------------------------ */
int dc_proton_raytrace(int gpu_id,
                       const float *rlsp, int nz, int ny, int nx,
                       const float spacing[3], const float origin[3],
                       const float iso[3], double gantry_deg, float couch_deg,
                       float vsadx, float vsady,
                       float *wet_out);

int dc_proton_raytrace_dev(int gpu_id,
                           const float *rlsp_dev, int nz, int ny, int nx,
                           const float spacing[3], const float origin[3],
                           const float iso[3], double gantry_deg, float couch_deg,
                           float vsadx, float vsady,
                           float *wet_out_dev, void *stream);

/* No counterpart in the reference.  Same result as dc_proton_raytrace_dev
 * (within the rounding of its interpolation weights) for callers that
 * cannot let the library allocate device memory: it allocates nothing.  Its
 * only scratch is a device array of 4,194,304 floats (16 MiB) inside the
 * library, held by every GPU that loads it until the process exits; larger
 * volumes are rejected with DC_ERR_VALUE.  The RLSP is read from the
 * caller's device buffer (no texture), the output goes to the caller's
 * device buffer, work is enqueued on `stream`.  The scratch is committed
 * on a device when the library's device code is loaded there, which under
 * CUDA's default lazy module loading is the first call on that device: that
 * call may fail with DC_ERR_CUDA (out of memory) on a full device, and it
 * looks up the scratch address, so make it before any stream capture (the
 * lookup is repeated once after a device reset).  The calling thread's
 * current device is restored on return.  All calls share the scratch:
 * calls that overlap on the GPU race. */
int dc_proton_raytrace_noalloc(int gpu_id,
                               const float *rlsp_dev, int nz, int ny, int nx,
                               const float spacing[3], const float origin[3],
                               const float iso[3], double gantry_deg, float couch_deg,
                               float vsadx, float vsady,
                               float *wet_out_dev, void *stream);

/* ------------------------------------------------------------------ */
/* Proton: double-Gaussian pencil-beam dose from a precomputed WET      */
/* Replaces dose_kernels.proton_spot_cuda                               */
/* (dosemodule.cu:243-374 -> IMPTClasses.cu:301-340).                   */
/*  divergence_params : [n_energies][dvp_len] = energy, R80, A, B, C    */
/*  lut_*             : [n_energies][lut_len] depth (mm), sigma (mm),   */
/*                      IDD; the reference uses lut_len = 400           */
/*  spots             : [n_spots][4] = x (mm), y (mm), MU, energy_id    */
/* Output: dose (Gy for the tables' calibration), accumulated over the  */
/* spots of the beam.                                                   */
/* ------------------------------------------------------------------ */
int dc_proton_spot(int gpu_id,
                   const float *wet, int nz, int ny, int nx,
                   const float spacing[3], const float origin[3],
                   const float iso[3], double gantry_deg, float couch_deg,
                   float vsadx, float vsady,
                   const float *divergence_params, int n_energies, int dvp_len,
                   const float *lut_depths, const float *lut_sigmas,
                   const float *lut_idds, int lut_len,
                   const float *spots, int n_spots,
                   float *dose_out);

/* Device variant.  wet/dose/LUT pointers are device pointers; `spots` is a
 * HOST array (the layer table is built on the host, as the reference does
 * in dosemodule.cu:204-225 and IMPTClasses.cu:37-67). */
int dc_proton_spot_dev(int gpu_id,
                       const float *wet_dev, int nz, int ny, int nx,
                       const float spacing[3], const float origin[3],
                       const float iso[3], double gantry_deg, float couch_deg,
                       float vsadx, float vsady,
                       const float *divergence_params, int n_energies, int dvp_len,
                       const float *lut_depths_dev, const float *lut_sigmas_dev,
                       const float *lut_idds_dev, int lut_len,
                       const float *spots, int n_spots,
                       float *dose_out_dev, void *stream);

/* ------------------------------------------------------------------ */
/* Proton beam kept on the device: dose from device-side spot weights,  */
/* the adjoint D^T g and the dose-influence matrix.  No counterpart in  */
/* the reference beyond its WET reuse (computeIMPTWET /                 */
/* computeIMPTPlanFromWET, plan_impt.py:162-211).  The handle holds the */
/* sorted spot/layer tables and the LUTs on its device; every call uses */
/* the same per-pair influence K_s(v) (dose per MU of spot s in voxel v)*/
/* as dc_proton_spot.  Spot-indexed arrays are in the order of `spots`. */
/* ------------------------------------------------------------------ */
typedef struct dc_proton_beam dc_proton_beam;

/* Arguments as dc_proton_spot, all host arrays (copied to the device). */
int dc_proton_beam_create(int gpu_id, int nz, int ny, int nx,
                          const float spacing[3], const float origin[3],
                          const float iso[3], double gantry_deg, float couch_deg,
                          float vsadx, float vsady,
                          const float *divergence_params, int n_energies, int dvp_len,
                          const float *lut_depths, const float *lut_sigmas,
                          const float *lut_idds, int lut_len,
                          const float *spots, int n_spots,
                          dc_proton_beam **out);
int dc_proton_beam_destroy(dc_proton_beam *beam);
int dc_proton_beam_info(const dc_proton_beam *beam, int *n_spots, int *n_layers, long long *n_voxels);

/* dose_dev[v] = sum_s mu_s K_s(v); mu_dev: n_spots floats on the device, or
 * NULL for the MU column of the spot list. */
int dc_proton_beam_dose(dc_proton_beam *beam, const float *wet_dev, const float *mu_dev,
                        float *dose_dev, void *stream);

/* grad_mu_dev[s] = sum_v grad_dose_dev[v] K_s(v) (FP64, overwritten). */
int dc_proton_beam_adjoint(dc_proton_beam *beam, const float *wet_dev, const float *grad_dose_dev,
                           double *grad_mu_dev, void *stream);
/* Voxel-list forms (no reference counterpart): the dose of the n voxels
 * listed in voxels_dev (flat indices into the beam's grid; entries outside
 * the grid give 0) into out_dev[0..n), and the adjoint of a gradient given
 * at those voxels only (grad_dev[0..n)) into grad_mu_dev (n_spots doubles,
 * overwritten).  The same per-pair influence as the volume forms; an
 * objective defined on a voxel subset (target, organs at risk) needs only
 * these.  A list sorted by voxel index keeps each CTA's voxels together. */
int dc_proton_beam_dose_list(dc_proton_beam *b, const float *wet_dev, const float *mu_dev, const int *voxels_dev,
                             int n, float *out_dev, void *stream);
int dc_proton_beam_adjoint_list(dc_proton_beam *b, const float *wet_dev, const int *voxels_dev, int n,
                                const float *grad_dev, double *grad_mu_dev, void *stream);

/* Influence matrix A (voxels x spots) in CSR with voxel rows: entries
 * K_s(v) >= cutoff * max_v K_s(v).  _nnz computes the entry count
 * (synchronises); _csr fills row_ptr_dev (n_voxels + 1, int64), col_dev
 * (spot index, int32) and val_dev (float32), writing at most `capacity`
 * entries. */
int dc_proton_beam_influence_nnz(dc_proton_beam *beam, const float *wet_dev, float cutoff,
                                 long long *nnz, void *stream);
int dc_proton_beam_influence_csr(dc_proton_beam *beam, const float *wet_dev, float cutoff,
                                 long long *row_ptr_dev, int *col_dev, float *val_dev,
                                 long long capacity, void *stream);

/* ------------------------------------------------------------------ */
/* Many IMPT plans in one persistent launch.  No counterpart in the     */
/* reference, which computes one beam per call (plan_impt.py:139-160).  */
/* Plans (CT grid, RLSP and dose volumes on the device) and beams       */
/* (geometry, host spot list, device WET volume) are added, then        */
/* committed (tables, work queues and textures are built); after that   */
/* the WET and dose calls only enqueue device work on `stream`, so they */
/* can be captured into a CUDA graph.  All beams share one beam model.  */
/* ------------------------------------------------------------------ */
typedef struct dc_proton_batch dc_proton_batch;

int dc_proton_batch_create(int gpu_id, const float *divergence_params, int n_energies, int dvp_len,
                           const float *lut_depths, const float *lut_sigmas, const float *lut_idds,
                           int lut_len, float vsadx, float vsady, dc_proton_batch **out);
int dc_proton_batch_add_plan(dc_proton_batch *batch, int nz, int ny, int nx, const float spacing[3],
                             const float origin[3], const float *rlsp_dev, float *dose_dev, int *plan_id);
int dc_proton_batch_add_beam(dc_proton_batch *batch, int plan_id, const float iso[3], double gantry_deg,
                             float couch_deg, const float *spots, int n_spots, float *wet_dev, int *beam_id);
int dc_proton_batch_commit(dc_proton_batch *batch);
/* n_variants: tile shapes the dose call accepts (for autotuning). */
int dc_proton_batch_info(const dc_proton_batch *batch, int *n_plans, int *n_beams, int *n_spots_total,
                         int *n_variants);
/* Offset of a beam's spots in the batch's spot-weight vector. */
int dc_proton_batch_beam_spot_offset(const dc_proton_batch *batch, int beam_id, int *offset);
/* WET (ray march + smoothing) of every beam into its WET volume. */
int dc_proton_batch_wet(dc_proton_batch *batch, void *stream);
/* Dose of every plan (sum of its beams) into its dose volume.  mu_dev:
 * n_spots_total weights on the device (beam by beam, each in its spot
 * list's order), or NULL to reuse the previous weights (initially the MU
 * column of the spot lists). */
int dc_proton_batch_dose(dc_proton_batch *batch, const float *mu_dev, int variant, void *stream);
/* Influence matrix of one beam (beam_id in add order; after
 * dc_proton_batch_wet), count-then-fill, one beam at a time so that memory
 * stays bounded by the largest beam's matrix.  Voxel rows of the beam's plan
 * grid, spot columns in the beam's spot-list order, entries K_s(v) >= cutoff
 * * max_v K_s(v) (the entries dc_proton_beam_influence_csr gives for the
 * same beam and WET).  _count writes the row starts (n_voxels + 1 int64)
 * into row_ptr_dev and the entry count into *nnz (synchronises); _fill
 * then writes col_dev (int32) and val_dev (float32, dose per MU) for the
 * beam _count ran last, capacity >= nnz.  No counterpart in the reference. */
int dc_proton_batch_influence_count(dc_proton_batch *batch, int beam_id, float cutoff, long long *row_ptr_dev,
                                    long long *nnz, void *stream);
int dc_proton_batch_influence_fill(dc_proton_batch *batch, int beam_id, const long long *row_ptr_dev, int *col_dev,
                                   float *val_dev, long long capacity, void *stream);
int dc_proton_batch_destroy(dc_proton_batch *batch);

/* ------------------------------------------------------------------ */
/* Photon: ray trace + TERMA + collapsed-cone convolution/superposition */
/* Replaces dose_kernels.photon_dose_cuda                               */
/* (dosemodule.cu:377-557 -> IMRTClasses.cu:353-405).                   */
/* Output: dose for one control point (before the output factor, which  */
/* the plan layer applies, plan_imrt.py:151-153).                       */
/* ------------------------------------------------------------------ */
int dc_photon_dose(int gpu_id,
                   const float *density, int nz, int ny, int nx,
                   const float spacing[3], const float origin[3],
                   const dc_photon_model *model, const dc_control_point *cp,
                   float *dose_out);

int dc_photon_dose_dev(int gpu_id,
                       const float *density_dev, int nz, int ny, int nx,
                       const float spacing[3], const float origin[3],
                       const dc_photon_model *model, const dc_control_point *cp,
                       float *dose_out_dev, void *stream);

/* ------------------------------------------------------------------ */
/* HU conversion on the device and device-resident plan loops.          */
/* They replace the host-side np.interp conversion and per-beam /        */
/* per-control-point loops of the plan layer (plan_impt.py:112-160,      */
/* plan_imrt.py:114-158) with the same arithmetic: the converted volume  */
/* equals np.interp(...).astype(float32) bit for bit, and the photon     */
/* accumulation is float32(acc + float64(dose) * weight).  Tables are    */
/* host arrays of n_table (<= 64) strictly increasing HU and the values. */
/* ------------------------------------------------------------------ */
int dc_hu_convert_dev(int gpu_id, const float *hu_dev, int nz, int ny, int nx, const double *table_hu,
                      const double *table_val, int n_table, float *out_dev, void *stream);
/* dc_proton_raytrace_dev from an HU volume: HU -> RLSP is written straight
 * into the ray tracer's texture array, then the WET march + smoothing. */
int dc_proton_raytrace_hu_dev(int gpu_id, const float *hu_dev, int nz, int ny, int nx, const float spacing[3],
                              const float origin[3], const double *table_hu, const double *table_rlsp, int n_table,
                              const float iso[3], double gantry_deg, float couch_deg, float vsadx, float vsady,
                              float *wet_out_dev, void *stream);
/* Several control points of one photon beam model in one call: the volume
 * (relative density, or HU converted with the table when is_hu) is loaded
 * once; for each control point dose_accum += weights[i] * CCCS dose
 * (weights: output factors, host doubles).  dose_accum is not cleared. */
int dc_photon_plan_dose_dev(int gpu_id, const float *volume_dev, int is_hu, const double *table_hu,
                            const double *table_density, int n_table, int nz, int ny, int nx, const float spacing[3],
                            const float origin[3], const dc_photon_model *model, const dc_control_point *cps,
                            int n_cps, const double *weights, float *dose_accum_dev, void *stream);

/* ------------------------------------------------------------------ */
/* Photon beam kept on the device (surrogate path).  No counterpart in  */
/* the reference: it splits dc_photon_dose into its TERMA pass and its  */
/* CCCS pass so that one TERMA serves the surrogate's input, a sparse   */
/* CCCS probe and, on rejection, the full CCCS.  Same kernels and       */
/* results as dc_photon_dose.  All volume pointers are device pointers. */
/* ------------------------------------------------------------------ */
typedef struct dc_photon_beam dc_photon_beam;

int dc_photon_beam_create(int gpu_id, int nz, int ny, int nx, const float spacing[3], const float origin[3],
                          dc_photon_beam **out);
int dc_photon_beam_destroy(dc_photon_beam *beam);
/* Copies the relative-density volume (device, (nz,ny,nx) float32). */
int dc_photon_beam_set_density(dc_photon_beam *beam, const float *density_dev, void *stream);
/* Ray trace + TERMA of one control point; terma_out_dev (or NULL)
 * receives the TERMA volume. */
int dc_photon_beam_terma(dc_photon_beam *beam, const dc_photon_model *model, const dc_control_point *cp,
                         float *terma_out_dev, void *stream);
/* Full CCCS dose of the last TERMA (as dc_photon_dose_dev). */
int dc_photon_beam_dose(dc_photon_beam *beam, float *dose_out_dev, void *stream);
/* No counterpart in the reference.  The CCCS of the beam's TERMA by
 * cone-direction sweeps (an approximation of cccKernel, IMRTClasses.cu:
 * 252-350): per cone direction, (TERMA, density) sampled once per node of a
 * lattice of parallel lines one voxel apart over the irradiated region, the
 * truncated recursions of every node from one warp-level scan along its line,
 * and the result interpolated at each voxel.  Drops the per-voxel kernel tilt
 * (:173-203) and interpolates between lines, so it is not held to the parity
 * bar; isotropic grids only.  Synchronises `stream` once. */
int dc_photon_beam_dose_sweep(dc_photon_beam *beam, float *dose_out_dev, void *stream);
/* Probe voxels of a control point: rays from the source through the open
 * field's centre, half-field and edge positions, lateral profiles at three
 * depths, and every lattice_stride-th voxel along each axis (0: no lattice;
 * default 4).  dc_photon_beam_terma selects them (on the host, while its
 * kernels run) and uploads them on its stream; probe_select repeats that. */
int dc_photon_beam_probe_config(dc_photon_beam *beam, int lattice_stride);
int dc_photon_beam_probe_select(dc_photon_beam *beam, int *n_out, void *stream);
/* The selected list: device pointer and count, and optionally a host copy
 * of the first `cap` indices. */
int dc_photon_beam_probe_list(const dc_photon_beam *beam, const int **voxels_dev, int *n, int *voxels_host, int cap);
/* CCCS dose at n listed voxels (voxels_dev NULL: the selected list). */
int dc_photon_beam_probe(dc_photon_beam *beam, const int *voxels_dev, int n, float *dose_out_dev, void *stream);

/* No counterpart in the reference (its TERMA has no fluence input,
 * IMRTClasses.cu:209-250).  A beamlet fluence map on the beam's-eye-view
 * isocentre plane (head frame: a along x, b along y, mm): beamlet (ia, ib)
 * at (a0 + ia*pitch, b0 + ib*pitch), values row-major [nb][na].  Each voxel's
 * TERMA and electron term of the last dc_photon_beam_terma are scaled by the
 * map's bilinear interpolation at the voxel's ray (clamped to the map's
 * edge), with the CCCS mask of the unmodulated TERMA, so the dose is linear
 * in the fluence; an all-ones map gives dc_photon_beam_dose bit for bit.
 * fluence_dose leaves the modulated TERMA in the beam (dose/probe then use
 * it); fluence_adjoint writes d(sum_v grad_dose_v D_v)/d fluence (float64,
 * one per beamlet), the transpose of the collapsed-cone superposition. */
typedef struct dc_fluence_map {
    int na, nb;
    float a0, b0, pitch;
} dc_fluence_map;
int dc_photon_beam_fluence_dose(dc_photon_beam *beam, const dc_fluence_map *map, const float *fluence_dev,
                                float *dose_out_dev, void *stream);
int dc_photon_beam_fluence_adjoint(dc_photon_beam *beam, const dc_fluence_map *map, const float *grad_dose_dev,
                                   double *grad_fluence_dev, void *stream);

/* Gamma index of the evaluated volume eval (nz,ny,nx) against reference
 * doses: ref[i] at voxel voxels[i] (i < n), or, with voxels NULL, the
 * reference volume ref.  Global dose criterion dd_frac*dose_norm (dose_norm
 * <= 0: the maximum of eval), distance dta_mm, reference points below
 * cutoff_frac*dose_norm skipped.  counts_dev[4]: [0] evaluated points,
 * [1] points with gamma <= 1, [2] scratch (all overwritten). */
int dc_gamma(int gpu_id, const float *eval_dev, int nz, int ny, int nx, const float spacing[3], const int *voxels_dev,
             const float *ref_dev, long long n, float dose_norm, float dta_mm, float dd_frac, float cutoff_frac,
             int *counts_dev, void *stream);

/* ------------------------------------------------------------------ */
/* Surrogate network building blocks (photon dose from TERMA+density). */
/* No counterpart in the reference, which has no learned model.         */
/* All pointers are device pointers on gpu_id; work is enqueued on      */
/* `stream` (NULL: legacy default stream) and nothing is synchronised.  */
/* Activations are bf16 (uint16 storage), channels-last (n,d,h,w,c).    */
/* Master weights are fp32:                                              */
/*   3x3x3 and 2x2x2-stride-2 convolutions: [taps][cin][cout],           */
/*     tap = (dz*k + dy)*k + dx;                                         */
/*   transposed 2x2x2 convolution: [8][cout][cin].                       */
/* Supported channel pairs: 3x3x3 8->16, 16->16, 32->32, 64->64,         */
/* 128->128; 2x2x2 stride 2 16->32, 32->64, 64->128; transposed          */
/* 32->16, 64->32, 128->64 (and their backward passes).                  */
/* ------------------------------------------------------------------ */
#define DC_NET_CONV3 0 /* 3x3x3, stride 1, zero padding 1 (same grid)  */
#define DC_NET_DOWN2 1 /* 2x2x2, stride 2 (grid halves)                 */

/* Number of 8-byte fragments of a packed weight set: ceil(taps*k/16) *
 * (n/8) * 32, where k is the reduction and n the output channel count. */
long long dc_net_packed_fragments(int taps, int k_per_tap, int n);

/* Packs master weights m[taps][a][b] into mma fragment order for a GEMM
 * with output channels n = (trans ? a : b) and reduction k = (trans ? b :
 * a) per tap; flip reverses the tap order (the 3x3x3 backward-data pass). */
int dc_net_pack_weights(int gpu_id, const float *master_dev, int taps, int a, int b, int flip, int trans,
                        void *packed_dev, void *stream);

/* Gather convolution y = conv(x) (mode DC_NET_CONV3 or DC_NET_DOWN2),
 * x: (n,d,h,w,cin), y on the output grid; wpk_frags: size of the packed
 * weights (must equal dc_net_packed_fragments(taps, cin, cout)).  stats (or
 * NULL): [n][cout][2] sum and sum of squares of the stored bf16 outputs
 * (overwritten). */
int dc_net_conv(int gpu_id, int mode, const void *x_dev, int n, int d, int h, int w, int cin, const void *wpk_dev,
                long long wpk_frags, int cout, void *y_dev, double *stats_dev, void *stream);

/* Transposed 2x2x2 stride-2 convolution y = up(x) + addend, x on the
 * coarse grid (n,d,h,w,cin), y on (n,2d,2h,2w,cout); addend may be NULL or
 * alias y. */
int dc_net_conv_up(int gpu_id, const void *x_dev, int n, int d, int h, int w, int cin, const void *wpk_dev,
                   long long wpk_frags, int cout, const void *addend_dev, void *y_dev, void *stream);

/* Weight gradient G[taps][ca][cb] = sum_o P[g(o,t)][a] Q[o][b] over the Q
 * grid (n,d,h,w,cb); P is on the same grid (DC_NET_CONV3, 27 taps) or on
 * the doubled grid (DC_NET_DOWN2, 8 taps).  grad is overwritten. */
int dc_net_wgrad(int gpu_id, int mode, const void *p_dev, const void *q_dev, int n, int d, int h, int w, int ca,
                 int cb, float *grad_dev, void *stream);

/* Instance norm: coef[n][c] = (gamma*rstd, beta - mean*gamma*rstd, mean,
 * rstd) from the statistics of dc_net_conv over `count` voxels. */
int dc_net_norm_finalize(int gpu_id, const double *stats_dev, int n, int c, long long count, const float *gamma_dev,
                         const float *beta_dev, float eps, float *coef_dev, void *stream);
/* a = leaky_relu(coef.x*y + coef.y, slope). */
int dc_net_norm_act(int gpu_id, const void *y_dev, int n, long long vox, int c, const float *coef_dev, float slope,
                    void *a_dev, void *stream);
/* dc_net_norm_finalize and dc_net_norm_act in one pass (n <= 16); coef_dev
 * (or NULL) receives the coefficients for the backward pass. */
int dc_net_norm_stats_act(int gpu_id, const void *y_dev, int n, long long vox, int c, const double *stats_dev,
                          long long count, const float *gamma_dev, const float *beta_dev, float eps, float slope,
                          float *coef_dev, void *a_dev, void *stream);
/* Backward of norm+activation: dy from da, and dgamma/dbeta (overwritten);
 * red: [n][c][2] double scratch. */
int dc_net_norm_act_bwd(int gpu_id, const void *y_dev, const void *da_dev, int n, long long vox, int c,
                        const float *coef_dev, const float *gamma_dev, float slope, double *red_dev, void *dy_dev,
                        float *dgamma_dev, float *dbeta_dev, void *stream);

/* The same 3x3x3 convolution on the 5th-generation tensor cores (tcgen05
 * MMA, fp32 accumulators in tensor memory) for grids of x extent 128 with
 * even y and z extents, 8->16 or 16->16 channels (the network's
 * full-resolution layers).  Weights are packed by dc_net_pack_weights_tc
 * into dc_net_packed_tc_bytes(cin, cout) bytes (-1: unsupported pair);
 * stats as dc_net_conv. */
long long dc_net_packed_tc_bytes(int cin, int cout);
int dc_net_pack_weights_tc(int gpu_id, const float *master_dev, int taps, int a, int b, int flip, int trans,
                           void *packed_dev, void *stream);
int dc_net_conv_tc(int gpu_id, const void *x_dev, int n, int d, int h, int w, int cin, const void *wtc_dev,
                   long long wtc_bytes, int cout, void *y_dev, double *stats_dev, void *stream);
/* Reads and clears the flag the tensor-core convolution sets when its
 * bounded wait for the tensor cores expired (that launch's output is not
 * written).  When it is set by a launch whose MMAs were issued (anything but
 * dc_net_tc_selftest, which withholds them), the expired CTA has released
 * tensor memory that those MMAs may still write, so every later result on
 * that device is suspect until the process recreates its CUDA context;
 * treat a set flag as a device error.  Synchronous. */
int dc_net_tc_error(int gpu_id, int *flag);
/* Failure self-test of that bounded wait: runs one tile with its MMAs
 * withheld, so the wait must expire; *wait_expired = 1 when the kernel
 * detected it and returned (the device stays usable).  Synchronous. */
int dc_net_tc_selftest(int gpu_id, int *wait_expired);

/* Network input: x8[v] = (terma*terma_scale, density, 0 x 6). */
int dc_net_pack_input(int gpu_id, const float *terma_dev, const float *density_dev, long long vox, float terma_scale,
                      void *x8_dev, void *stream);
/* Output head (16 channels -> 1): out = mask > mask_thr ?
 * scale*(w.g + bias) : 0. */
int dc_net_head(int gpu_id, const void *g_dev, long long vox, int c, const float *w_dev, const float *bias_dev,
                const float *mask_dev, float mask_thr, float scale, float *out_dev, void *stream);
/* Squared-error loss over voxels with target >= 0, times inv_count (read
 * from inv_count_dev instead when that is not NULL, e.g. inside a CUDA
 * graph), and its gradients: dg (16 channels), dw, dbias, loss (all
 * overwritten). */
int dc_net_head_loss_bwd(int gpu_id, const void *g_dev, long long vox, int c, const float *w_dev,
                         const float *pred_dev, const float *target_dev, float inv_count,
                         const float *inv_count_dev, double *loss_dev, void *dg_dev, float *dw_dev,
                         float *dbias_dev, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* DOSECUDA_H */
