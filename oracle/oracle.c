/*
 * oracle.c — CPU restatement of the reference DoseCUDA dose engines, used as
 * TEST INFRASTRUCTURE ONLY (the checker and the CPU baseline).  Nothing in the
 * product links or calls it.
 *
 * Arithmetic policy ("FP64 values, reference-float decisions"):
 *  - Every quantity that decides discrete control flow in the reference —
 *    sample positions and texture coordinates and the volume-exit test of the
 *    ray march, nearest-voxel rounding in the WET smoothing, the LUT bracket
 *    search, the layer range cut, the CCCS sample counts, the TERMA mask —
 *    is evaluated in float32 with the reference's expression order
 *    (fmaf where the reference writes fmaf), so both pick the same samples.
 *  - Every physical value (texture interpolation, WET sums, LUT
 *    interpolation, Gaussians, erf/exp, recursions, dose sums) is computed
 *    in double.
 *  - Texture sampling restates CUDA's documented linear filtering of a
 *    border-addressed 3D texture with unnormalised coordinates: x -= 0.5,
 *    i = floor(x), alpha = frac(x), trilinear blend of the 8 neighbours with
 *    the border value outside the volume.  tex_mode 0 uses exact weights;
 *    tex_mode 1 quantises alpha to 8 fractional bits (the CUDA Programming
 *    Guide's texture-fetching appendix stores the weights in 9-bit fixed
 *    point with 8 fractional bits).
 *
 * Reference functions restated (paths within the DoseCUDA project):
 *   rayTraceKernel        DoseCUDA/dose_kernels/CudaClasses.cu:180-228
 *   CudaBeam geometry     CudaClasses.cu:17-126, CudaClasses.cuh:41-52,96-116
 *   smoothRayKernel       DoseCUDA/dose_kernels/IMPTClasses.cu:139-202
 *   importLayers + sort   IMPTClasses.cu:37-67, dosemodule.cu:204-225
 *   pencilBeamKernel      IMPTClasses.cu:204-271 (+ :69-133 helpers)
 *   termaKernel           DoseCUDA/dose_kernels/IMRTClasses.cu:209-250 (+ :120-171)
 *   cccKernel             IMRTClasses.cu:252-350 (+ kernelTilt :173-203)
 *   Texture3D sampler     DoseCUDA/dose_kernels/TextureClasses.cu:5-38
 *
 * Build: oracle/build.py (gcc -O2 -fopenmp -ffp-contract=off).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define PI_F 3.14159265358979323846f
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#define AIR_DENSITY 0.0012f

typedef struct { float x, y, z; } f3;
typedef struct { double x, y, z; } d3;

typedef struct {
    int nx, ny, nz;
    float sx, sy, sz, ix, iy, iz; /* spacing and its float reciprocal */
} grid_t;

typedef struct {
    float isox, isoy, isoz, srcx, srcy, srcz;
    float sga, cga, sta, cta, sca, cca;
} frame_t;

/* ---------------------------------------------------------------- geometry */
static grid_t make_grid(int nz, int ny, int nx, const float sp[3]) {
    grid_t g;
    g.nx = nx; g.ny = ny; g.nz = nz;
    g.sx = sp[0]; g.sy = sp[1]; g.sz = sp[2];
    g.ix = 1.0f / g.sx; g.iy = 1.0f / g.sy; g.iz = 1.0f / g.sz;
    return g;
}

/* CudaBeam ctor (CudaClasses.cu:17-51), gantry offset (dosemodule.cu:152). */
static frame_t make_frame(const float iso[3], const float origin[3], double gantry, double couch,
                          double coll, float src_dist) {
    frame_t f;
    f.isox = iso[0] - origin[0];
    f.isoy = iso[1] - origin[1];
    f.isoz = iso[2] - origin[2];
    float ga = fmodf((float)(gantry + 180.0f), 360.0f) * PI_F / 180.0f;
    float ta = (float)couch * PI_F / 180.0f;
    float ca = (float)coll * PI_F / 180.0f;
    f.sga = sinf(ga); f.cga = cosf(ga);
    f.sta = sinf(ta); f.cta = cosf(ta);
    f.sca = sinf(ca); f.cca = cosf(ca);
    float xg = -src_dist * f.sga, yg = src_dist * f.cga;
    f.srcx = xg * f.cta;
    f.srcy = yg;
    f.srcz = -xg * f.sta;
    return f;
}

static f3 voxel_xyz(const grid_t *g, const frame_t *f, int i, int j, int k) {
    f3 p;
    p.x = (float)i * g->sx - f->isox;
    p.y = (float)j * g->sy - f->isoy;
    p.z = (float)k * g->sz - f->isoz;
    return p;
}

static f3 tex_coord(const grid_t *g, const frame_t *f, f3 p) {
    f3 t;
    t.x = fmaf(g->ix, p.x + f->isox, 0.5f);
    t.y = fmaf(g->iy, p.y + f->isoy, 0.5f);
    t.z = fmaf(g->iz, p.z + f->isoz, 0.5f);
    return t;
}

static int tex_inside(const grid_t *g, f3 t) {
    return t.x >= 0.0f && t.x < (float)g->nx && t.y >= 0.0f && t.y < (float)g->ny && t.z >= 0.0f &&
           t.z < (float)g->nz;
}

static f3 unit_to_source_f(const frame_t *f, f3 p) {
    f3 u = {f->srcx - p.x, f->srcy - p.y, f->srcz - p.z};
    float r = (float)(1.0 / sqrt((double)u.x * u.x + (double)u.y * u.y + (double)u.z * u.z));
    u.x *= r; u.y *= r; u.z *= r;
    return u;
}

static d3 unit_to_source_d(const frame_t *f, d3 p) {
    d3 u = {f->srcx - p.x, f->srcy - p.y, f->srcz - p.z};
    double r = 1.0 / sqrt(u.x * u.x + u.y * u.y + u.z * u.z);
    u.x *= r; u.y *= r; u.z *= r;
    return u;
}

/* image -> head (CudaClasses.cu:65-95; IMRTClasses.cu:41-79 with collimator) */
static f3 image_to_head_f(const frame_t *f, f3 p, int coll) {
    float s = -f->sta, c = f->cta;
    float xt = p.x * c + p.z * s, yt = p.y, zt = -p.x * s + p.z * c;
    s = -f->sga; c = f->cga;
    float xg = xt * c - yt * s, yg = xt * s + yt * c, zg = zt;
    if (coll) {
        s = -f->sca; c = f->cca;
        float xc = xg * c + zg * s, zc = -xg * s + zg * c;
        xg = xc; zg = zc;
    }
    f3 h = {-xg, zg, yg};
    return h;
}

static d3 image_to_head_d(const frame_t *f, d3 p, int coll) {
    double s = -f->sta, c = f->cta;
    double xt = p.x * c + p.z * s, yt = p.y, zt = -p.x * s + p.z * c;
    s = -f->sga; c = f->cga;
    double xg = xt * c - yt * s, yg = xt * s + yt * c, zg = zt;
    if (coll) {
        s = -f->sca; c = f->cca;
        double xc = xg * c + zg * s, zc = -xg * s + zg * c;
        xg = xc; zg = zc;
    }
    d3 h = {-xg, zg, yg};
    return h;
}

/* head -> image (CudaClasses.cu:97-126; IMRTClasses.cu:81-118) */
static f3 head_to_image_f(const frame_t *f, f3 h, int coll) {
    float x = -h.x, y = h.z, z = h.y, s, c;
    if (coll) {
        s = f->sca; c = f->cca;
        float xc = x * c + z * s, zc = -x * s + z * c;
        x = xc; z = zc;
    }
    s = f->sga; c = f->cga;
    float xg = x * c - y * s, yg = x * s + y * c, zg = z;
    s = f->sta; c = f->cta;
    f3 r = {xg * c + zg * s, yg, -xg * s + zg * c};
    return r;
}

static d3 head_to_image_d(const frame_t *f, d3 h, int coll) {
    double x = -h.x, y = h.z, z = h.y, s, c;
    if (coll) {
        s = f->sca; c = f->cca;
        double xc = x * c + z * s, zc = -x * s + z * c;
        x = xc; z = zc;
    }
    s = f->sga; c = f->cga;
    double xg = x * c - y * s, yg = x * s + y * c, zg = z;
    s = f->sta; c = f->cta;
    d3 r = {xg * c + zg * s, yg, -xg * s + zg * c};
    return r;
}

static int lower_bound_f(const float *d, int n, float key) {
    int l = 0, r = n;
    while (l < r) {
        int m = (l + r) / 2;
        if (key <= d[m]) r = m; else l = m + 1;
    }
    return l;
}

/* ------------------------------------------------------------ texture model */
static double texel(const float *v, const grid_t *g, long i, long j, long k, double border) {
    if (i < 0 || j < 0 || k < 0 || i >= g->nx || j >= g->ny || k >= g->nz) return border;
    return (double)v[i + (long)g->nx * (j + (long)g->ny * k)];
}

static double frac_weight(double a, int mode) {
    if (mode == 1) return nearbyint(a * 256.0) / 256.0;
    return a;
}

/* Linear-filtered, border-addressed fetch at unnormalised coordinates. */
static double tex_fetch(const float *v, const grid_t *g, double x, double y, double z, double border, int mode) {
    x -= 0.5; y -= 0.5; z -= 0.5;
    double fx = floor(x), fy = floor(y), fz = floor(z);
    long i = (long)fx, j = (long)fy, k = (long)fz;
    double a = frac_weight(x - fx, mode), b = frac_weight(y - fy, mode), c = frac_weight(z - fz, mode);
    double r = 0.0;
    for (int dk = 0; dk < 2; ++dk)
        for (int dj = 0; dj < 2; ++dj)
            for (int di = 0; di < 2; ++di) {
                double w = (di ? a : 1.0 - a) * (dj ? b : 1.0 - b) * (dk ? c : 1.0 - c);
                if (w != 0.0) r += w * texel(v, g, i + di, j + dj, k + dk, border);
            }
    return r;
}

/* ------------------------------------------------------------- WET march */
/* rayTraceKernel (CudaClasses.cu:180-228); returns WET in cm. */
static double wet_ray(const float *rho, const grid_t *g, const frame_t *f, int i, int j, int k, double border,
                      int mode, long *n_samples) {
    f3 p = voxel_xyz(g, f, i, j, k);
    f3 u = unit_to_source_f(f, p);
    double wet = -0.05;
    long n = 0;
    for (float t = 0.0f;; t += 1.0f) {
        f3 q = {fmaf(u.x, t, p.x), fmaf(u.y, t, p.y), fmaf(u.z, t, p.z)};
        f3 tc = tex_coord(g, f, q);
        if (!tex_inside(g, tc)) break;
        double d = tex_fetch(rho, g, tc.x, tc.y, tc.z, border, mode);
        wet += 0.1 * (d > 0.0 ? d : 0.0);
        ++n;
    }
    if (n_samples) *n_samples += n;
    return wet;
}

/* Proton WET ray trace + BEV smoothing (IMPTClasses.cu:139-202, 274-299).
 * wet_raw (optional) receives the unsmoothed WET; wet the smoothed one (cm).
 * Returns the number of texture samples taken by the march. */
long oracle_proton_wet(const float *rlsp, int nz, int ny, int nx, const float spacing[3], const float origin[3],
                       const float iso[3], double gantry, float couch, float vsadx, float vsady, int tex_mode,
                       double *wet_raw, double *wet) {
    grid_t g = make_grid(nz, ny, nx, spacing);
    frame_t f = make_frame(iso, origin, gantry, couch, 0.0, (vsadx + vsady) / 2.0f);
    long n = (long)nx * ny * nz;
    double *raw = wet_raw ? wet_raw : (double *)malloc(sizeof(double) * n);
    float *rawf = (float *)malloc(sizeof(float) * n);
    long total = 0;
#pragma omp parallel for collapse(2) schedule(dynamic, 4) reduction(+ : total)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                long v = i + (long)nx * (j + (long)ny * k);
                raw[v] = wet_ray(rlsp, &g, &f, i, j, k, 0.0, tex_mode, &total);
                rawf[v] = (float)raw[v];
            }
    if (wet) {
#pragma omp parallel for collapse(2) schedule(static)
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    long v = i + (long)nx * (j + (long)ny * k);
                    f3 p = voxel_xyz(&g, &f, i, j, k);
                    f3 h = image_to_head_f(&f, p, 0);
                    float c = rawf[v];
                    double sum = raw[v];
                    int cnt = 1;
                    for (int d = 0; d < 6; ++d) {
                        /* sincosf((float)d * PI / 3) of the reference, in double then rounded */
                        float ang = (float)d * PI_F / 3.0f;
                        float s = (float)sin((double)ang), co = (float)cos((double)ang);
                        for (float dr = 1.0f; dr < c * 10.0f && dr < 10.0f; dr += 1.0f) {
                            f3 hc = {h.x + dr * co, h.y + dr * s, h.z};
                            f3 q = head_to_image_f(&f, hc, 0);
                            int qi = (int)roundf((q.x + f.isox) / g.sx);
                            int qj = (int)roundf((q.y + f.isoy) / g.sy);
                            int qk = (int)roundf((q.z + f.isoz) / g.sz);
                            if (qi >= 0 && qj >= 0 && qk >= 0 && qi < nx && qj < ny && qk < nz) {
                                sum += raw[qi + (long)nx * (qj + (long)ny * qk)];
                                ++cnt;
                            }
                        }
                    }
                    wet[v] = sum / cnt;
                }
    }
    free(rawf);
    if (!wet_raw) free(raw);
    return total;
}

/* ------------------------------------------------------------- pencil beam */
typedef struct {
    int e;
    int order;
    float x, y, mu;
} spot_t;

static int spot_cmp(const void *a, const void *b) {
    const spot_t *p = (const spot_t *)a, *q = (const spot_t *)b;
    if (p->e != q->e) return p->e < q->e ? -1 : 1;
    return p->order < q->order ? -1 : (p->order > q->order);
}

/* pencilBeamKernel (IMPTClasses.cu:204-271).  `wet` is the smoothed WET (cm)
 * as the reference receives it (float).  Returns the number of
 * (voxel, spot) pairs evaluated (voxels inside the layer's range), or -1 on
 * an invalid energy id. */
static long g_last_near_pairs = 0;

long oracle_proton_dose(const float *wet, int nz, int ny, int nx, const float spacing[3], const float origin[3],
                        const float iso[3], double gantry, float couch, float vsadx, float vsady,
                        const float *dvp, int n_energies, int dvp_len, const float *lut_d, const float *lut_s,
                        const float *lut_i, int lut_len, const float *spots, int n_spots, double *dose) {
    grid_t g = make_grid(nz, ny, nx, spacing);
    frame_t f = make_frame(iso, origin, gantry, couch, 0.0, (vsadx + vsady) / 2.0f);
    spot_t *sp = (spot_t *)malloc(sizeof(spot_t) * (n_spots > 0 ? n_spots : 1));
    for (int s = 0; s < n_spots; ++s) {
        float e = spots[4 * s + 3];
        if (!(e > -1.0f) || !(e < (float)n_energies)) {
            free(sp);
            return -1;
        }
        sp[s].e = (int)e;
        sp[s].order = s;
        sp[s].x = spots[4 * s];
        sp[s].y = spots[4 * s + 1];
        sp[s].mu = spots[4 * s + 2];
    }
    qsort(sp, n_spots, sizeof(spot_t), spot_cmp);
    /* layers */
    int *ls = (int *)malloc(sizeof(int) * (n_spots + 1));
    int nl = 0;
    for (int s = 0; s < n_spots; ++s)
        if (s == 0 || sp[s].e != sp[s - 1].e) ls[nl++] = s;
    ls[nl] = n_spots;
    long pairs = 0, near = 0;
    double VX = vsadx, VY = vsady;
#pragma omp parallel for collapse(2) schedule(dynamic, 2) reduction(+ : pairs, near)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                long v = i + (long)nx * (j + (long)ny * k);
                float w_mm = wet[v] * 10.0f;
                f3 pf = voxel_xyz(&g, &f, i, j, k);
                d3 p = {pf.x, pf.y, pf.z};
                d3 h = image_to_head_d(&f, p, 0);
                double dsrc = sqrt((f.srcx - p.x) * (f.srcx - p.x) + (f.srcy - p.y) * (f.srcy - p.y) +
                                   (f.srcz - p.z) * (f.srcz - p.z));
                double total = 0.0;
                for (int l = 0; l < nl; ++l) {
                    int e = sp[ls[l]].e;
                    const float *row = dvp + (long)dvp_len * e;
                    float r80f = row[1];
                    if (w_mm > 1.1f * r80f) continue;
                    double r80 = r80f, w = w_mm;
                    const float *D = lut_d + (long)e * lut_len, *S = lut_s + (long)e * lut_len,
                                *I = lut_i + (long)e * lut_len;
                    int q = lower_bound_f(D, lut_len, w_mm);
                    double idd, sig;
                    if (q == lut_len) { idd = I[q - 1]; sig = S[q - 1]; }
                    else if (q == 0) { idd = I[0]; sig = S[0]; }
                    else {
                        double fac = (w - D[q - 1]) / ((double)D[q] - D[q - 1]);
                        idd = I[q - 1] + ((double)I[q] - I[q - 1]) * fac;
                        sig = S[q - 1] + ((double)S[q] - S[q - 1]) * fac;
                    }
                    double d = dsrc - w + 0.7 * r80;
                    double st = ((double)row[2] * d + row[3]) * d + row[4] + sig;
                    double wc = w < 0.1 ? 0.1 : w;
                    double hi = r80 - 0.1;
                    if (wc > hi) wc = hi;
                    double hs = 2.85 + 0.0014 * r80 * log(wc + 3.0) + 0.06 * wc - 7.4e-5 * wc * wc -
                                (0.22 * r80) / ((wc - r80 - 5.0) * (wc - r80 - 5.0));
                    double hw = 0.052 * log(1.13 + wc / (11.2 - 0.023 * r80)) +
                                0.35 * (0.0017 * r80 * r80 - r80) / ((r80 + 3.0) * (r80 + 3.0) - wc * wc) -
                                1.61e-9 * wc * (r80 + 3.0) * (r80 + 3.0);
                    if (hs < 0.0) hs = 0.0;
                    if (hw < 0.0) hw = 0.0;
                    if (hw > 0.9) hw = 0.9;
                    double sht = sqrt(st * st + hs * hs);
                    double pfac = (1.0 - hw) * idd / (2.0 * M_PI * st * st);
                    double hfac = hw * idd / (2.0 * M_PI * sht * sht);
                    double ps = -0.5 / (st * st), hsc = -0.5 / (sht * sht);
                    double acc = 0.0, reach2 = 36.0 * sht * sht;
                    for (int s = ls[l]; s < ls[l + 1]; ++s) {
                        double tx = sp[s].x / VX, ty = sp[s].y / VY;
                        double rx = h.x - sp[s].x, ry = h.y - sp[s].y, rz = h.z;
                        double t2 = tx * tx + ty * ty + 1.0;
                        double ray2 = rx * rx + ry * ry + rz * rz;
                        double dot = tx * rx + ty * ry - rz;
                        double r2 = ray2 - dot * dot / t2;
                        acc += sp[s].mu * (pfac * exp(ps * r2) + hfac * exp(hsc * r2));
                        near += r2 <= reach2;
                    }
                    pairs += ls[l + 1] - ls[l];
                    total += acc;
                }
                dose[v] = total;
            }
    free(ls);
    free(sp);
    g_last_near_pairs = near;
    return pairs;
}

/* (voxel, spot) pairs of the last oracle_proton_dose call whose distance from
 * the spot's axis is within 6 halo sigmas at the voxel (6 * sqrt(sigma_tot^2 +
 * sigma_halo^2)): the pencil beam's work unit inside its cut-off radius. */
long oracle_last_near_pairs(void) { return g_last_near_pairs; }

/* ------------------------------------------------------------- photon */
typedef struct {
    int n_prof;
    const float *prof_r, *prof_i, *prof_s;
    int n_spec;
    const float *spec_mu, *spec_pw, *spec_sw;
    float mu_cal, psd, ssd, pss, sss, mlc_dist, ssw, ea, esw, efd;
    int n_cones;
    const float *k_theta, *k_Am, *k_am, *k_Bm, *k_bm, *k_rl;
} photon_model_t;

typedef struct {
    int n_pairs;
    const float *x1, *x2, *yoff, *yw;
} mlc_t;

/* headTransmission (IMRTClasses.cu:120-150) */
static double head_transmission(const photon_model_t *m, const mlc_t *mlc, d3 p, double iso_to_src, double sigma) {
    double scale = ((double)m->psd - m->mlc_dist) / m->psd;
    double div = (iso_to_src - p.z) / (m->mlc_dist - p.z);
    double k = 1.0 / (sigma * sqrt(2.0));
    double t = 0.0;
    for (int q = 0; q < mlc->n_pairs; ++q) {
        double yb = (mlc->yoff[q] - 0.5 * mlc->yw[q]) * scale, yt = (mlc->yoff[q] + 0.5 * mlc->yw[q]) * scale;
        double xl = mlc->x1[q] * scale, xr = mlc->x2[q] * scale;
        double t1 = (xl - p.x) * div + p.x, t2 = (xr - p.x) * div + p.x;
        double e1 = (yb - p.y) * div + p.y, e2 = (yt - p.y) * div + p.y;
        t += 0.5 * (erf(t2 * k) - erf(t1 * k)) * 0.5 * (erf(e2 * k) - erf(e1 * k));
    }
    return t;
}

/* Primary and scatter head transmission at every voxel centre
 * (headTransmission, IMRTClasses.cu:120-150, as called by termaKernel
 * :209-250), in double.  Tests use it to locate voxels whose primary
 * transmission vanishes, where the reference's TERMA divides by it. */
void oracle_photon_transmission(int nz, int ny, int nx, const float spacing[3], const float origin[3],
                                const photon_model_t *m, const float iso[3], double gantry, float coll, float couch,
                                const mlc_t *mlc, double *tp_out, double *ts_out) {
    grid_t g = make_grid(nz, ny, nx, spacing);
    frame_t f = make_frame(iso, origin, gantry, couch, coll, m->psd);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                long v = i + (long)nx * (j + (long)ny * k);
                f3 pf = voxel_xyz(&g, &f, i, j, k);
                d3 p = {pf.x, pf.y, pf.z};
                d3 h = image_to_head_d(&f, p, 1);
                tp_out[v] = head_transmission(m, mlc, h, m->psd, m->pss);
                ts_out[v] = head_transmission(m, mlc, h, m->ssd, m->sss);
            }
}

/* Photon dose of one control point (IMRTClasses.cu:209-405).  terma/electron
 * (optional) receive the intermediate volumes.  Returns the number of CCCS
 * samples (2 texture fetches each) taken. */
long oracle_photon_dose(const float *density, int nz, int ny, int nx, const float spacing[3], const float origin[3],
                        const photon_model_t *m, const float iso[3], float mu, double gantry, float coll,
                        float couch, const mlc_t *mlc, int tex_mode, double *terma_out, double *electron_out,
                        double *dose) {
    grid_t g = make_grid(nz, ny, nx, spacing);
    frame_t f = make_frame(iso, origin, gantry, couch, coll, m->psd);
    long n = (long)nx * ny * nz;
    double *wet = (double *)malloc(sizeof(double) * n);
    double *terma = terma_out ? terma_out : (double *)malloc(sizeof(double) * n);
    double *elec = electron_out ? electron_out : (double *)malloc(sizeof(double) * n);
    float *termaf = (float *)malloc(sizeof(float) * n);
#pragma omp parallel for collapse(2) schedule(dynamic, 4)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                long v = i + (long)nx * (j + (long)ny * k);
                wet[v] = wet_ray(density, &g, &f, i, j, k, AIR_DENSITY, tex_mode, NULL);
            }
    /* TERMA */
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                long v = i + (long)nx * (j + (long)ny * k);
                f3 pf = voxel_xyz(&g, &f, i, j, k);
                d3 p = {pf.x, pf.y, pf.z};
                d3 h = image_to_head_d(&f, p, 1);
                double dp = m->psd - h.z, ds = m->ssd - h.z;
                double rc = sqrt(h.x * h.x + h.y * h.y) * (m->psd - h.z) / m->psd;
                double oaf, soft;
                int q = lower_bound_f(m->prof_r, m->n_prof, (float)rc);
                if (q == m->n_prof) { oaf = m->prof_i[q - 1]; soft = m->prof_s[q - 1]; }
                else if (q == 0) { oaf = m->prof_i[0]; soft = m->prof_s[0]; }
                else {
                    double mm = (rc - m->prof_r[q - 1]) / ((double)m->prof_r[q] - m->prof_r[q - 1]);
                    oaf = m->prof_i[q - 1] + ((double)m->prof_i[q] - m->prof_i[q - 1]) * mm;
                    soft = m->prof_s[q - 1] + ((double)m->prof_s[q] - m->prof_s[q - 1]) * mm;
                }
                double tp = head_transmission(m, mlc, h, m->psd, m->pss);
                double ts = head_transmission(m, mlc, h, m->ssd, m->sss);
                double w = (float)wet[v];
                double ratio = ts / tp;
                if (!(ratio < 1.0)) ratio = 1.0; /* fminf(1, x): NaN and inf give 1 */
                double tsum = 0.0;
                for (int e = 0; e < m->n_spec; ++e) {
                    double att = exp(-(double)m->spec_mu[e] * w * soft);
                    tsum += (1.0 - ratio) * (m->spec_pw[e] * att * (m->psd / dp) * (m->psd / dp)) +
                            ratio * m->spec_sw[e] * att * (m->ssd / ds);
                }
                double ed = exp(-(double)m->ea * m->efd);
                double el = (exp(-(double)m->ea * w) - ed) / (1.0 - ed);
                if (el < 0.0) el = 0.0;
                terma[v] = oaf * ((1.0 - m->ssw) * tp * tsum + m->ssw * ts * tsum);
                termaf[v] = (float)terma[v];
                elec[v] = m->esw * (0.4 + 0.3 * ratio) * el * tp;
            }
    /* cones: sample distances (float sequence, IMRTClasses.cu:313-333) */
    float sp_cm = g.sx / 10.0f;
    int off[16], cnt[16];
    float rl10[1024];
    int tot = 0;
    for (int c = 0; c < m->n_cones && c < 16; ++c) {
        off[c] = tot;
        cnt[c] = 0;
        for (float rl = m->k_rl[c]; rl >= 0.0f && tot < 1024; rl = rl - sp_cm) {
            rl10[tot++] = rl * 10.0f;
            cnt[c]++;
        }
    }
    /* 72 head-frame directions rotated to the image frame (voxel independent) */
    d3 dirs[16 * 12];
    double sth_c[16];
    for (int c = 0; c < m->n_cones && c < 16; ++c) {
        double th = (double)m->k_theta[c] * M_PI / 180.0;
        sth_c[c] = sin(th);
        for (int a = 0; a < 12; ++a) {
            double phi = a * M_PI / 6.0;
            d3 th_head = {sin(th) * cos(phi), sin(th) * sin(phi), cos(th)};
            dirs[c * 12 + a] = head_to_image_d(&f, th_head, 1);
        }
    }
    d3 zero = {0, 0, 0};
    d3 axis0 = unit_to_source_d(&f, zero);
    long samples = 0;
#pragma omp parallel for collapse(2) schedule(dynamic, 1) reduction(+ : samples)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                long v = i + (long)nx * (j + (long)ny * k);
                f3 pf = voxel_xyz(&g, &f, i, j, k);
                f3 tc0 = tex_coord(&g, &f, pf);
                if ((float)tex_fetch(termaf, &g, tc0.x, tc0.y, tc0.z, 0.0, tex_mode) <= 0.01f) {
                    dose[v] = 0.0;
                    continue;
                }
                d3 p = {pf.x, pf.y, pf.z};
                d3 u = unit_to_source_d(&f, p);
                double costh = axis0.x * u.x + axis0.y * u.y + axis0.z * u.z;
                d3 ax = {axis0.y * u.z - axis0.z * u.y, axis0.z * u.x - axis0.x * u.z, axis0.x * u.y - axis0.y * u.x};
                double dv = 0.0;
                for (int c = 0; c < m->n_cones; ++c) {
                    double Am = m->k_Am[c], am = m->k_am[c], Bm = m->k_Bm[c], bm = m->k_bm[c];
                    double sth = sth_c[c];
                    for (int a = 0; a < 12; ++a) {
                        d3 t = dirs[c * 12 + a];
                        d3 r = {ax.y * t.z - ax.z * t.y, ax.z * t.x - ax.x * t.z, ax.x * t.y - ax.y * t.x};
                        double sc = (ax.x * t.x + ax.y * t.y + ax.z * t.z) / (1.0 + costh);
                        r.x += t.x * costh + ax.x * sc;
                        r.y += t.y * costh + ax.y * sc;
                        r.z += t.z * costh + ax.z * sc;
                        double Rp = 0.0, Rs = 0.0;
                        for (int s = 0; s < cnt[c]; ++s) {
                            double L = rl10[off[c] + s];
                            double qx = p.x + r.x * L, qy = p.y + r.y * L, qz = p.z + r.z * L;
                            double tx = (qx + f.isox) / g.sx + 0.5, ty = (qy + f.isoy) / g.sy + 0.5,
                                   tz = (qz + f.isoz) / g.sz + 0.5;
                            double T = tex_fetch(termaf, &g, tx, ty, tz, 0.0, tex_mode);
                            double D = tex_fetch(density, &g, tx, ty, tz, AIR_DENSITY, tex_mode);
                            if (D < AIR_DENSITY) D = AIR_DENSITY;
                            D *= sp_cm;
                            double ex = exp(-am * D);
                            Rp = Rp * ex + T * sth * (Am / (am * am)) * (1.0 - ex);
                            Rs = Rs * (1.0 - bm * D) + T * D * sth * (Bm / bm);
                        }
                        samples += cnt[c];
                        dv += am * Rp + bm * Rs;
                    }
                }
                dv += elec[v];
                dose[v] = (dv == dv && dv >= 0.0) ? (double)m->mu_cal * dv * mu : 0.0;
            }
    free(termaf);
    free(wet);
    if (!terma_out) free(terma);
    if (!electron_out) free(elec);
    return samples;
}

int oracle_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
