// dc_common.cuh — grid and beam geometry shared by the DoseCUDA B200 kernels.
//
// The coordinate conventions follow the reference engine exactly, because the
// dose depends on where every texture sample lands:
//  * voxel (i,j,k) sits at xyz = ijk*spacing - iso_rel, where iso_rel is the
//    isocentre relative to the volume origin (CudaClasses.cuh:106-110,
//    dosemodule.cu:160-164);
//  * texture coordinates are (xyz + iso_rel)/spacing + 0.5
//    (CudaClasses.cuh:100-104), inside while 0 <= t < n (:90-94);
//  * the source sits at distance SAD from the isocentre after the gantry
//    (about z) and couch (about y) rotations (CudaClasses.cu:17-51);
//  * image <-> head (nozzle/BEV) frames are the couch, gantry and, for
//    photons, collimator rotations (CudaClasses.cu:65-126,
//    IMRTClasses.cu:41-118).
// The float expressions keep the reference's operation order where a
// rounding difference could move a sample across a texel or volume boundary
// (positions, texture coordinates, nearest-voxel rounding); elsewhere the
// kernels are free to reorder.
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

// Debug builds (-DDC_DEBUG_BOUNDS; `python -m dosecuda_b200.build
// --debug-bounds --out PATH`) check the index of each instrumented global
// access against its buffer's extent.  The first violation in a translation
// unit is recorded in that unit's error word (site << 48 | index & 2^48-1)
// and the access is skipped, so an indexing bug shows up as a report
// (dc_debug_bounds) instead of a fault.  Release builds compile the checks
// away: DC_IN_BOUNDS is the constant true.
#ifdef DC_DEBUG_BOUNDS
#define DC_BOUNDS_WORD static __device__ unsigned long long g_dc_bounds = 0ull;
__device__ __forceinline__ bool dc_in_bounds_impl(unsigned long long *word, long long idx, long long n,
                                                  unsigned site) {
    if (idx >= 0 && idx < n) return true;
    atomicCAS(word, 0ull, ((unsigned long long)site << 48) | ((unsigned long long)idx & 0xFFFFFFFFFFFFull));
    return false;
}
#define DC_IN_BOUNDS(idx, n, site) \
    ::dc_in_bounds_impl(&g_dc_bounds, (long long)(idx), (long long)(n), (unsigned)(site))
#define DC_BOUNDS_TAKE(fn)                                                          \
    unsigned long long fn() {                                                       \
        unsigned long long v = 0ull, z = 0ull;                                      \
        if (cudaMemcpyFromSymbol(&v, g_dc_bounds, sizeof(v)) != cudaSuccess) v = ~0ull; \
        cudaMemcpyToSymbol(g_dc_bounds, &z, sizeof(z));                             \
        return v;                                                                   \
    }
#else
#define DC_BOUNDS_WORD
#define DC_IN_BOUNDS(idx, n, site) true
#define DC_BOUNDS_TAKE(fn) \
    unsigned long long fn() { return 0ull; }
#endif

namespace dc {

constexpr float kAirDensity = 0.0012f;  // g/cc, IMRTClasses.cuh:6

// Regular grid.  Array shape (nz, ny, nx); index i + nx*(j + ny*k).
struct Grid {
    int nx, ny, nz;
    float sx, sy, sz;           // spacing, mm
    float inv_sx, inv_sy, inv_sz;  // 1/spacing (IEEE-rounded, as 1.0f/sp on device)
    __host__ __device__ long long n() const { return (long long)nx * ny * nz; }
};

// Beam geometry: isocentre (relative to the volume origin), source position
// relative to the isocentre, cached trig of the machine angles.
struct Frame {
    float isox, isoy, isoz;
    float srcx, srcy, srcz;
    float sga, cga;   // gantry (after the +180 degree offset)
    float sta, cta;   // couch
    float sca, cca;   // collimator (0 for protons)
};

// ---------------------------------------------------------------------------
// Host-side construction (reference CudaBeam ctor, CudaClasses.cu:17-51;
// collimator trig IMRTClasses.cu:30-39; gantry offset dosemodule.cu:152).
// ---------------------------------------------------------------------------
Frame make_frame(const float iso[3], const float origin[3], double gantry_deg,
                 double couch_deg, double collimator_deg, float src_dist);
Grid make_grid(int nz, int ny, int nx, const float spacing[3]);

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ float3 voxel_xyz(const Grid &g, const Frame &f, int i, int j, int k) {
    float3 p;
    p.x = (float)i * g.sx - f.isox;
    p.y = (float)j * g.sy - f.isoy;
    p.z = (float)k * g.sz - f.isoz;
    return p;
}

__device__ __forceinline__ float3 tex_coord(const Grid &g, const Frame &f, float3 p) {
    float3 t;
    t.x = fmaf(g.inv_sx, p.x + f.isox, 0.5f);
    t.y = fmaf(g.inv_sy, p.y + f.isoy, 0.5f);
    t.z = fmaf(g.inv_sz, p.z + f.isoz, 0.5f);
    return t;
}

__device__ __forceinline__ bool tex_inside(const Grid &g, float3 t) {
    return t.x >= 0.0f && t.x < (float)g.nx && t.y >= 0.0f && t.y < (float)g.ny &&
           t.z >= 0.0f && t.z < (float)g.nz;
}

// Unit vector from p towards the source (CudaClasses.cuh:41-52).
__device__ __forceinline__ float3 unit_to_source(const Frame &f, float3 p) {
    float3 u = make_float3(f.srcx - p.x, f.srcy - p.y, f.srcz - p.z);
    const float r = rnorm3df(u.x, u.y, u.z);
    u.x *= r;
    u.y *= r;
    u.z *= r;
    return u;
}

__device__ __forceinline__ float distance_to_source(const Frame &f, float3 p) {
    return norm3df(f.srcx - p.x, f.srcy - p.y, f.srcz - p.z);
}

// Image -> head frame: couch, then gantry, then (photons) collimator, then the
// DICOM nozzle axis swap (CudaClasses.cu:65-95, IMRTClasses.cu:41-79).
template <bool kCollimator>
__host__ __device__ __forceinline__ float3 image_to_head(const Frame &f, float3 p) {
    float s = -f.sta, c = f.cta;
    const float xt = p.x * c + p.z * s;
    const float yt = p.y;
    const float zt = -p.x * s + p.z * c;
    s = -f.sga;
    c = f.cga;
    float xg = xt * c - yt * s;
    const float yg = xt * s + yt * c;
    float zg = zt;
    if (kCollimator) {
        s = -f.sca;
        c = f.cca;
        const float xc = xg * c + zg * s;
        const float zc = -xg * s + zg * c;
        xg = xc;
        zg = zc;
    }
    return make_float3(-xg, zg, yg);
}

// Head -> image frame, the inverse sequence (CudaClasses.cu:97-126,
// IMRTClasses.cu:81-118).
template <bool kCollimator>
__host__ __device__ __forceinline__ float3 head_to_image(const Frame &f, float3 h) {
    float x = -h.x;
    float y = h.z;
    float z = h.y;
    float s, c;
    if (kCollimator) {
        s = f.sca;
        c = f.cca;
        const float xc = x * c + z * s;
        const float zc = -x * s + z * c;
        x = xc;
        z = zc;
    }
    s = f.sga;
    c = f.cga;
    const float xg = x * c - y * s;
    const float yg = x * s + y * c;
    const float zg = z;
    s = f.sta;
    c = f.cta;
    float3 r;
    r.x = xg * c + zg * s;
    r.y = yg;
    r.z = -xg * s + zg * c;
    return r;
}

// First index i in [0, n] with key <= data[i] (CudaClasses.cuh:130-144).
__host__ __device__ __forceinline__ int lower_bound(const float *data, int n, float key) {
    int l = 0, r = n;
    while (l < r) {
        const int mid = (l + r) >> 1;
        if (key <= data[mid]) {
            r = mid;
        } else {
            l = mid + 1;
        }
    }
    return l;
}

__device__ __forceinline__ float sqr(float x) { return x * x; }

__device__ __forceinline__ float clampf(float x, float lo, float hi) {
    return fminf(fmaxf(x, lo), hi);
}

// 2^x on the special-function unit (PTX ex2.approx.ftz.f32; relative error
// about 2^-22, flushes results below 2^-126 to zero).
__device__ __forceinline__ float fast_exp2(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

constexpr float kLog2e = 1.4426950408889634f;

}  // namespace dc
