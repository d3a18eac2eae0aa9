/*
 * fd_oracle.c -- CPU restatement of the reference path (TEST INFRASTRUCTURE).
 *
 * This is the checker the CUDA kernels of fastdose_b200 are compared against and
 * the timed CPU baseline; the product never calls it.  The arithmetic type of
 * the dose math is FD_REAL (double for the parity build, float for the timed
 * build).  Host geometry is float, as the reference's host code is.
 *
 * Parity quirks of the reference reproduced here:
 *   Q1 d_calcg uses integer division, so g == 1 (DoseComp.cu:167-175).
 *   Q2 cumu_p_i is reset inside the phi loop, so a slice is normalised by the
 *      last azimuth's path sum only (DoseComp.cu:321,389).
 *   Q3 the reset of SharedDose / cumu_p_i is modelled as happening before any
 *      accumulation into them (DoseComp.cu:311,321,364-365).
 *   Q4 lateral wrap-around with the X recursion reset on crossing
 *      (DoseComp.cu:147-164,372-377).
 * Texture sampling: tex_mode 0 uses exact trilinear weights; tex_mode 1 rounds
 * them to 1/256 like the texture unit's 8-bit fraction.
 */
#include "fd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef FD_REAL
#define FD_REAL double
#endif
typedef FD_REAL real;

#define EPS_FD 1e-4f          /* eps_fastdose, FastDoseLib/include/macros.h:21 */
#define LARGER_EPS_FD 1e-3f   /* larger_eps_fastdose, macros.h:22 */
#define PI_F 3.14159265358979323846f

/* ------------------------------------------------------------ float geometry */

/* rotateAroundAxisAtOriginRHS, FastDoseLib/src/geom.cu:11-34 (Rodrigues). */
void or_rotate_axis_f(const float p[3], const float r[3], float t, float out[3]) {
    float s = sinf(t), c = cosf(t);
    float omc = 1.0f - c;
    float pr = p[0] * r[0] + p[1] * r[1] + p[2] * r[2];
    float k = omc * pr;
    float o0 = k * r[0] + c * p[0] + s * (r[1] * p[2] - r[2] * p[1]);
    float o1 = k * r[1] + c * p[1] + s * (r[2] * p[0] - r[0] * p[2]);
    float o2 = k * r[2] + c * p[2] + s * (r[0] * p[1] - r[1] * p[0]);
    out[0] = o0; out[1] = o1; out[2] = o2;
}

/* rotateBeamAtOriginRHS (PVCS -> BEV), geom.cu:36-44. */
void or_rotate_beam_f(const float v[3], float theta, float phi, float coll, float out[3]) {
    float axis[3] = {sinf(-phi), 0.0f, cosf(-phi)};
    float tmp[3];
    or_rotate_axis_f(v, axis, -theta, tmp);
    float yaxis[3] = {0.0f, 1.0f, 0.0f};
    or_rotate_axis_f(tmp, yaxis, phi + coll, out);
}

/* inverseRotateBeamAtOriginRHS (BEV -> PVCS), geom.cu:47-56. */
void or_inv_rotate_beam_f(const float v[3], float theta, float phi, float coll, float out[3]) {
    float yaxis[3] = {0.0f, 1.0f, 0.0f};
    float tmp[3];
    or_rotate_axis_f(v, yaxis, -(phi + coll), tmp);
    float axis[3] = {sinf(-phi), 0.0f, cosf(-phi)};
    or_rotate_axis_f(tmp, axis, theta, out);
}

static float f3len(const float v[3]) { return sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }
static float f3dot(const float a[3], const float b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
/* Reciprocal square root rounded once from the exact value (evaluated in
 * double); the reference's host normalize()/rsqrt produce these same values. */
static float rsqrt_cr(float x) { return (float)(1.0 / sqrt((double)x)); }
static void f3normalize(float v[3]) {
    float inv = rsqrt_cr(f3dot(v, v));
    v[0] *= inv; v[1] *= inv; v[2] *= inv;
}

/* BEAM_h::calc_range, FastDoseLib/src/beam.cu:134-222 (quirk Q5 kept: corner 2
 * uses half_fluence_size.x for its z component; the running max starts at
 * FLT_MIN). */
int or_calc_range(fd2_beam_t* b, const fd2_volume_t* vol) {
    float hx = b->fmap_size[0] * b->beamlet_size[0] / 2;
    float hy = b->fmap_size[1] * b->beamlet_size[1] / 2;
    float bnd[5][3] = {
        {hx, b->sad, hy}, {hx, b->sad, -hy}, {-hx, b->sad, hx}, {-hx, b->sad, -hy}, {0, b->sad, 0}};
    for (int i = 0; i < 5; i++) {
        float t[3];
        or_inv_rotate_beam_f(bnd[i], b->angles[0], b->angles[1], b->angles[2], t);
        bnd[i][0] = t[0]; bnd[i][1] = t[1]; bnd[i][2] = t[2];
    }
    float src0[3] = {0.0f, -b->sad, 0.0f}, src[3];
    or_inv_rotate_beam_f(src0, b->angles[0], b->angles[1], b->angles[2], src);
    for (int j = 0; j < 3; j++) src[j] = src[j] + b->isocenter[j];
    for (int j = 0; j < 3; j++) b->source[j] = src[j];

    float bb0[3], bb1[3];
    for (int j = 0; j < 3; j++) {
        bb0[j] = (float)vol->bbox_start[j] * vol->voxel_size[j];
        bb1[j] = (float)(vol->bbox_start[j] + vol->bbox_dim[j]) * vol->voxel_size[j];
    }
    float dmin = 3.402823466e+38f;  /* numeric_limits<float>::max() */
    float dmax = 1.175494351e-38f;  /* numeric_limits<float>::min() (Q5) */
    int hit = 0;
    for (int i = 0; i < 5; i++) {
        const float* bd = bnd[i];
        float inter[6][3];
        for (int j = 0; j < 3; j++) {
            double denom = bd[j];
            denom = signbit(denom) ? denom - EPS_FD : denom + EPS_FD;
            double a1 = (bb0[j] - src[j]) / denom;
            double a2 = (bb1[j] - src[j]) / denom;
            for (int c = 0; c < 3; c++) {
                /* float3 + double * float3: helper_math promotes the scalar to float */
                inter[2 * j][c] = src[c] + (float)a1 * bd[c];
                inter[2 * j + 1][c] = src[c] + (float)a2 * bd[c];
            }
        }
        for (int j = 0; j < 3; j++) {
            for (int k = 0; k < 2; k++) {
                const float* it = inter[2 * j + k];
                int j1 = (j + 1) % 3, j2 = (j + 2) % 3;
                if (it[j1] >= bb0[j1] && it[j1] <= bb1[j1] && it[j2] >= bb0[j2] && it[j2] <= bb1[j2]) {
                    float d[3] = {it[0] - src[0], it[1] - src[1], it[2] - src[2]};
                    float len = f3len(d) * b->sad / f3len(bd);
                    dmin = fminf(len, dmin);
                    dmax = fmaxf(len, dmax);
                    hit = 1;
                }
            }
        }
    }
    if (!hit) return FD2_ERR_GEOMETRY;
    b->lim_min = dmin;
    b->lim_max = dmax;
    b->long_dim = (uint32_t)ceil((b->lim_max - b->lim_min) / b->long_spacing);
    return 0;
}

/* IMRT::BeamBundle::beamletInit, IMRTOpt/src/IMRTBeamBundle.cu:341-569. */
int or_beamlet_init(const fd2_bundle_t* bb, int ix, int iy, const fd2_volume_t* vol,
                    fd2_beam_t* out) {
    float hfx = bb->fluence_dim[0] * bb->beamlet_size[0] * 0.5f;
    float hfy = bb->fluence_dim[1] * bb->beamlet_size[1] * 0.5f;
    float v0[3] = {ix * bb->beamlet_size[0] - hfx, bb->sad, iy * bb->beamlet_size[1] - hfy};
    float v1[3] = {(ix + 1) * bb->beamlet_size[0] - hfx, bb->sad, iy * bb->beamlet_size[1] - hfy};
    float v2[3] = {(ix + 1) * bb->beamlet_size[0] - hfx, bb->sad, (iy + 1) * bb->beamlet_size[1] - hfy};
    float v3[3] = {ix * bb->beamlet_size[0] - hfx, bb->sad, (iy + 1) * bb->beamlet_size[1] - hfy};
    f3normalize(v0); f3normalize(v1); f3normalize(v2); f3normalize(v3);
    const float* vs[4] = {v0, v1, v2, v3};

    /* two candidate centre lines: bisector of (v0, v2) and of (v1, v3) */
    float cl[2][3], dist[2], proj[2][4][3];
    for (int cs = 0; cs < 2; cs++) {
        const float* a = cs == 0 ? v0 : v1;
        const float* c = cs == 0 ? v2 : v3;
        float l[3] = {a[0] + c[0], a[1] + c[1], a[2] + c[2]};
        f3normalize(l);
        cl[cs][0] = l[0]; cl[cs][1] = l[1]; cl[cs][2] = l[2];
        float d4[4];
        for (int q = 0; q < 4; q++) {
            float dd = f3dot(vs[q], l);
            for (int k = 0; k < 3; k++) proj[cs][q][k] = vs[q][k] / dd;
            float diff[3] = {proj[cs][q][0] - l[0], proj[cs][q][1] - l[1], proj[cs][q][2] - l[2]};
            d4[q] = f3len(diff);
        }
        if (cs == 0) {
            if (fabsf(d4[0] - d4[2]) > EPS_FD) return FD2_ERR_GEOMETRY;
            dist[0] = fminf(fminf(d4[0], d4[1]), d4[3]);
        } else {
            if (fabsf(d4[1] - d4[3]) > EPS_FD) return FD2_ERR_GEOMETRY;
            dist[1] = fminf(fminf(d4[0], d4[1]), d4[2]);
        }
    }
    int cs = dist[0] > dist[1] ? 0 : 1;
    float* dir = cl[cs];
    float p0[3], p1[3];
    for (int k = 0; k < 3; k++) {
        p0[k] = proj[cs][0][k] - dir[k];
        p1[k] = proj[cs][1][k] - dir[k];
    }
    f3normalize(p0); f3normalize(p1);
    float codir[3];
    if (cs == 0) {
        /* the reference adds vertex0_plane to itself here (IMRTBeamBundle.cu:425) */
        codir[0] = p0[0] + p0[0]; codir[1] = p0[1] + p0[1]; codir[2] = p0[2] + p0[2];
    } else {
        codir[0] = p0[0] + p1[0]; codir[1] = p0[1] + p1[1]; codir[2] = p0[2] + p1[2];
    }
    f3normalize(codir);
    float sad_r = bb->sad / dir[1];
    float hh[3], hw[3];
    for (int k = 0; k < 3; k++) {
        hh[k] = (p0[k] + p1[k]) * dist[cs] * 0.5f;
        hw[k] = (p0[k] - p1[k]) * dist[cs] * 0.5f;
    }
    float fl_h = f3len(hh) * sad_r * 2;
    float fl_w = f3len(hw) * sad_r * 2;

    float dpv[3];
    or_inv_rotate_beam_f(dir, bb->angles[0], bb->angles[1], bb->angles[2], dpv);
    float yax[3] = {0.0f, 1.0f, 0.0f};
    float theta = acosf(f3dot(dpv, yax));
    float smp = dpv[2] * rsqrt_cr(dpv[2] * dpv[2] + dpv[0] * dpv[0] + EPS_FD * EPS_FD);
    float phi = asinf(smp);

    float cand_t[4] = {theta, theta, -theta, -theta};
    float cand_p[4] = {phi, PI_F - phi, phi, PI_F - phi};
    int found = -1;
    for (int q = 0; q < 4; q++) {
        float r[3];
        or_inv_rotate_beam_f(yax, cand_t[q], cand_p[q], 0.0f, r);
        if (!(f3dot(r, dpv) < 1 - EPS_FD)) { found = q; break; }
    }
    if (found < 0) return FD2_ERR_GEOMETRY;
    float th_r = cand_t[found], ph_r = cand_p[found];

    float cdpv[3];
    or_inv_rotate_beam_f(codir, bb->angles[0], bb->angles[1], bb->angles[2], cdpv);
    float cbev[3] = {0.0f, 0.0f, -1.0f}, cir[3];
    or_inv_rotate_beam_f(cbev, th_r, ph_r, 0.0f, cir);
    float cosc = f3dot(cdpv, cir);
    cosc = cosc < -1.0f ? -1.0f : (cosc > 1.0f ? 1.0f : cosc);
    float coll = acosf(cosc);
    float coll_r = coll;
    or_inv_rotate_beam_f(cbev, th_r, ph_r, coll_r, cir);
    if (f3dot(cir, cdpv) < 1 - EPS_FD * 10) {
        coll_r = -coll;
        or_inv_rotate_beam_f(cbev, th_r, ph_r, coll_r, cir);
        if (f3dot(cir, cdpv) < 1 - EPS_FD * 10) return FD2_ERR_GEOMETRY;
    }

    memset(out, 0, sizeof(*out));
    out->angles[0] = th_r; out->angles[1] = ph_r; out->angles[2] = coll_r;
    float disp[3] = {(ix + 0.5f - 0.5f * bb->fluence_dim[0]) * bb->beamlet_size[0], 0.0f,
                     (iy + 0.5f - 0.5f * bb->fluence_dim[1]) * bb->beamlet_size[1]};
    float dpv2[3];
    or_inv_rotate_beam_f(disp, bb->angles[0], bb->angles[1], bb->angles[2], dpv2);
    for (int k = 0; k < 3; k++) out->isocenter[k] = bb->isocenter[k] + dpv2[k];
    out->beamlet_size[0] = fl_w / bb->sub_fluence_on[0];
    out->beamlet_size[1] = fl_h / bb->sub_fluence_on[1];
    out->fmap_size[0] = (uint32_t)bb->sub_fluence_dim[0];
    out->fmap_size[1] = (uint32_t)bb->sub_fluence_dim[1];
    out->sad = sad_r;
    out->long_spacing = bb->long_spacing;
    size_t pitch = (size_t)out->fmap_size[0] * out->fmap_size[1] * sizeof(float);
    out->TermaBEV_pitch = pitch;
    out->DensityBEV_pitch = pitch;
    return or_calc_range(out, vol);
}

/* Sub-beam fluence: centred sub_fluence_on^2 open square (IMRTBeamBundle.cu:553-563). */
void or_beamlet_fluence(const fd2_bundle_t* bb, float* out) {
    int fx = bb->sub_fluence_dim[0], fy = bb->sub_fluence_dim[1];
    memset(out, 0, sizeof(float) * fx * fy);
    int lx = (int)((fx - bb->sub_fluence_on[0]) * 0.5f);
    int ly = (int)((fy - bb->sub_fluence_on[1]) * 0.5f);
    for (int j = ly; j < ly + bb->sub_fluence_on[1]; j++)
        for (int i = lx; i < lx + bb->sub_fluence_on[0]; i++) out[i + j * fx] = 1.0f;
}

/* ------------------------------------------------------------ real geometry */
typedef struct { real x, y, z; } r3;

static void rot_axis(const real p[3], const real r[3], real t, real out[3]) {
    real s = sin(t), c = cos(t);
    real k = (1 - c) * (p[0] * r[0] + p[1] * r[1] + p[2] * r[2]);
    real o0 = k * r[0] + c * p[0] + s * (r[1] * p[2] - r[2] * p[1]);
    real o1 = k * r[1] + c * p[1] + s * (r[2] * p[0] - r[0] * p[2]);
    real o2 = k * r[2] + c * p[2] + s * (r[0] * p[1] - r[1] * p[0]);
    out[0] = o0; out[1] = o1; out[2] = o2;
}

/* 3x3 matrices of the two beam rotations, built once per beam (the rotation is
 * linear, so M*v equals the reference's two Rodrigues rotations up to rounding). */
static void beam_matrices(const fd2_beam_t* b, real fwd[9], real inv[9]) {
    for (int c = 0; c < 3; c++) {
        real e[3] = {0, 0, 0}, o[3], t[3];
        e[c] = 1;
        real th = b->angles[0], ph = b->angles[1], co = b->angles[2];
        real axis[3] = {sin(-ph), 0, cos(-ph)};
        real yax[3] = {0, 1, 0};
        rot_axis(e, axis, -th, t);
        rot_axis(t, yax, ph + co, o);
        for (int r = 0; r < 3; r++) fwd[r * 3 + c] = o[r];
        rot_axis(e, yax, -(ph + co), t);
        rot_axis(t, axis, th, o);
        for (int r = 0; r < 3; r++) inv[r * 3 + c] = o[r];
    }
}
static void mv(const real m[9], const real v[3], real o[3]) {
    real a = m[0] * v[0] + m[1] * v[1] + m[2] * v[2];
    real b = m[3] * v[0] + m[4] * v[1] + m[5] * v[2];
    real c = m[6] * v[0] + m[7] * v[1] + m[8] * v[2];
    o[0] = a; o[1] = b; o[2] = c;
}

static real qweight(real a, int tex_mode) {
    if (tex_mode == 1) return floor(a * 256 + (real)0.5) / 256;
    return a;
}

/* Linear-filtered, unnormalised, border-0 3-D texture fetch (texel centres at i+0.5). */
static real tex_linear(const float* v, int nx, int ny, int nz, real u, real w, real s, int tm) {
    real xb = u - (real)0.5, yb = w - (real)0.5, zb = s - (real)0.5;
    real fi = floor(xb), fj = floor(yb), fk = floor(zb);
    real ax = qweight(xb - fi, tm), ay = qweight(yb - fj, tm), az = qweight(zb - fk, tm);
    long i0 = (long)fi, j0 = (long)fj, k0 = (long)fk;
    real acc = 0;
    for (int dk = 0; dk < 2; dk++) {
        long k = k0 + dk;
        real wk = dk ? az : 1 - az;
        if (k < 0 || k >= nz || wk == 0) continue;
        for (int dj = 0; dj < 2; dj++) {
            long j = j0 + dj;
            real wj = dj ? ay : 1 - ay;
            if (j < 0 || j >= ny || wj == 0) continue;
            for (int di = 0; di < 2; di++) {
                long i = i0 + di;
                real wi = di ? ax : 1 - ax;
                if (i < 0 || i >= nx || wi == 0) continue;
                acc += wi * wj * wk * (real)v[i + (size_t)nx * (j + (size_t)ny * k)];
            }
        }
    }
    return acc;
}

/* ------------------------------------------------------------ beamlet flags */
/* d_beamletFlagInit, IMRTOpt/src/IMRTBeamBundle.cu:269-316: a fluence pixel is
 * on iff any of super_sampling^2 sub-rays, at any slice, samples the linear-
 * filtered PTV mask above 0. */
void or_beamlet_flags(size_t n_beams, const fd2_beam_t* beams, const uint8_t* ptv,
                      const fd2_volume_t* vol, int ss, int tex_mode, uint8_t* flags) {
    size_t nvox = (size_t)vol->dim[0] * vol->dim[1] * vol->dim[2];
    float* mask = (float*)malloc(nvox * sizeof(float));
    for (size_t i = 0; i < nvox; i++) mask[i] = (float)ptv[i];
#pragma omp parallel for schedule(dynamic)
    for (long bi = 0; bi < (long)n_beams; bi++) {
        const fd2_beam_t* b = &beams[bi];
        real fwd[9], inv[9];
        beam_matrices(b, fwd, inv);
        int fx = b->fmap_size[0], fy = b->fmap_size[1];
        for (int p = 0; p < fx * fy; p++) {
            int bx = p % fx, by = p / fx;
            int on = 0;
            for (uint32_t i = 0; i < b->long_dim && !on; i++) {
                real sxd = (real)b->lim_min + (real)i * b->long_spacing;
                for (int j = 0; j < ss && !on; j++) {
                    for (int k = 0; k < ss && !on; k++) {
                        real d[3] = {(bx + (j + (real)0.5) / ss - fx * (real)0.5) * b->beamlet_size[0],
                                     b->sad,
                                     (by + (k + (real)0.5) / ss - fy * (real)0.5) * b->beamlet_size[1]};
                        real pv[3];
                        mv(inv, d, pv);
                        real c[3];
                        for (int q = 0; q < 3; q++)
                            c[q] = ((real)b->source[q] + pv[q] * sxd / b->sad) / vol->voxel_size[q];
                        real val = tex_linear(mask, vol->dim[0], vol->dim[1], vol->dim[2], c[0], c[1],
                                              c[2], tex_mode);
                        if (val > 0) on = 1;
                    }
                }
            }
            flags[bi * (size_t)fx * fy + p] = (uint8_t)on;
        }
    }
    free(mask);
}

/* ------------------------------------------------------------ Terma */
#define SUPER_SAMPLING 4  /* TermaComp.cu:65 */

void or_terma(const fd2_beam_t* b, const float* fluence, const float* density,
              const fd2_volume_t* vol, int nkern, const float* energy, const float* sfl,
              const float* mu, int tex_mode, float* terma, float* dens) {
    real fwd[9], inv[9];
    beam_matrices(b, fwd, inv);
    int fx = b->fmap_size[0], fy = b->fmap_size[1];
    int P = fx * fy;
    size_t pitch = b->TermaBEV_pitch ? b->TermaBEV_pitch / sizeof(float) : (size_t)P;
#pragma omp parallel for schedule(dynamic)
    for (int p = 0; p < P; p++) {
        int ix = p % fx, iy = p / fx;
        real fl = fluence[p];
        real pc[3] = {(ix + (real)0.5 - fx * (real)0.5) * b->beamlet_size[0], b->sad,
                      (iy + (real)0.5 - fy * (real)0.5) * b->beamlet_size[1]};
        real pv[3];
        mv(inv, pc, pv);
        real k = (real)b->long_spacing / ((real)b->sad * SUPER_SAMPLING);
        real st[3] = {pv[0] * k, pv[1] * k, pv[2] * k};
        real stn = sqrt(st[0] * st[0] + st[1] * st[1] + st[2] * st[2]);
        real sxd = (real)b->lim_min / b->sad;
        real sxd_step = k;
        real cn[3], sn[3];
        for (int q = 0; q < 3; q++) {
            cn[q] = ((real)b->source[q] + pv[q] * sxd) / vol->voxel_size[q];
            sn[q] = st[q] / vol->voxel_size[q];
        }
        real rpl = 0;
        for (uint32_t i = 0; i < b->long_dim; i++) {
            real tavg = 0, davg = 0;
            for (int j = 0; j < SUPER_SAMPLING; j++) {
                cn[0] += sn[0]; cn[1] += sn[1]; cn[2] += sn[2];
                real d = tex_linear(density, vol->dim[0], vol->dim[1], vol->dim[2], cn[0], cn[1], cn[2],
                                    tex_mode);
                rpl += d * stn;
                davg += d;
                real tl = 0;
                for (int e = 0; e < nkern; e++) {
                    real f = (real)sfl[e] * fl;
                    tl += f * (real)energy[e] * (real)mu[e] * exp(-(real)mu[e] * rpl);
                }
                sxd += sxd_step;
                tavg += tl / (sxd * sxd);
            }
            terma[p + pitch * i] = (float)(tavg / SUPER_SAMPLING);
            dens[p + pitch * i] = (float)(davg / SUPER_SAMPLING);
        }
    }
}

/* ------------------------------------------------------------ CCCS */
/* d_nextPoint (device version), DoseComp.cu:76-111: step to the next voxel
 * boundary, snapping to the z plane when it lands within 1e-4 of it.  Float,
 * correctly-rounded division and fused multiply-add: the CUDA kernel performs
 * the same operations, so both make identical boundary decisions. */
void or_next_point_f(const float c[3], const float d[3], float out[3], int* flag) {
    float st[3];
    for (int q = 0; q < 3; q++) {
        if (d[q] == 0.0f)
            st[q] = INFINITY;  /* a still axis never limits the step */
        else if (d[q] > 0)
            st[q] = (ceilf(c[q] + LARGER_EPS_FD) - c[q]) / d[q];
        else
            st[q] = (floorf(c[q] - LARGER_EPS_FD) - c[q]) / d[q];
    }
    float take = fminf(fminf(st[0], st[1]), st[2]);
    float r[3] = {fmaf(take, d[0], c[0]), fmaf(take, d[1], c[1]), fmaf(take, d[2], c[2])};
    int f = fabsf(r[2] - roundf(r[2])) < EPS_FD;
    if (f) {
        take = st[2];
        r[0] = fmaf(take, d[0], c[0]);
        r[1] = fmaf(take, d[1], c[1]);
        r[2] = roundf(fmaf(take, d[2], c[2]));
    }
    out[0] = r[0]; out[1] = r[1]; out[2] = r[2];
    *flag = f;
}

void or_next_point(const double c[3], const double d[3], double out[3], int* flag) {
    float cf[3] = {(float)c[0], (float)c[1], (float)c[2]}, df[3] = {(float)d[0], (float)d[1], (float)d[2]};
    float of[3];
    or_next_point_f(cf, df, of, flag);
    out[0] = of[0]; out[1] = of[1]; out[2] = of[2];
}

/* d_calcLineSeg, DoseComp.cu:114-144: physical length of a segment given in
 * normalised BEV coordinates, lateral axes scaled by the divergence factor. */
double or_calc_line_seg(const double s[3], const double e[3], const fd2_beam_t* b) {
    double sp[3] = {(s[0] - b->fmap_size[0] * 0.5) * b->beamlet_size[0],
                    (s[1] - b->fmap_size[1] * 0.5) * b->beamlet_size[1], s[2] * b->long_spacing};
    double f = (sp[2] + b->lim_min) / b->sad;
    sp[0] *= f; sp[1] *= f;
    double ep[3] = {(e[0] - b->fmap_size[0] * 0.5) * b->beamlet_size[0],
                    (e[1] - b->fmap_size[1] * 0.5) * b->beamlet_size[1], e[2] * b->long_spacing};
    f = (ep[2] + b->lim_min) / b->sad;
    ep[0] *= f; ep[1] *= f;
    double dx = ep[0] - sp[0], dy = ep[1] - sp[1], dz = ep[2] - sp[2];
    return sqrt(dx * dx + dy * dy + dz * dz);
}

/* Cone direction in normalised BEV units (DoseComp.cu:280-290): the physical
 * direction (sin t cos p, sin t sin p, cos t) divided by the voxel size per axis
 * and normalised.  Evaluated in double and rounded to float, on the host, in
 * both this oracle and the library, so the ray geometry starts from identical
 * bits. */
void or_cone_direction(const fd2_beam_t* b, float theta, float phi, float out[3]) {
    double st = sin((double)theta), ct = cos((double)theta), sp = sin((double)phi), cp = cos((double)phi);
    double v[3] = {st * cp / b->beamlet_size[0], st * sp / b->beamlet_size[1], ct / b->long_spacing};
    double n = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    out[0] = (float)(v[0] / n); out[1] = (float)(v[1] / n); out[2] = (float)(v[2] / n);
}

void or_cccs(const fd2_beam_t* b, const float* terma, const float* dens, int n_theta,
             const float* theta, const float* A, const float* a, const float* B, const float* bb,
             int n_phi, const float* phi, float* dose) {
    or_cccs_dirs(b, terma, dens, n_theta, theta, A, a, B, bb, n_phi, phi, NULL, dose);
}

/* As or_cccs; when `given` is not NULL it holds the cone directions
 * [forward zenith bin][azimuth][4] to march with instead of or_cone_direction's. */
void or_cccs_dirs(const fd2_beam_t* b, const float* terma, const float* dens, int n_theta,
                  const float* theta, const float* A, const float* a, const float* B, const float* bb,
                  int n_phi, const float* phi, const float* given, float* dose) {
    int fx = b->fmap_size[0], fy = b->fmap_size[1];
    int t_fwd = 0;
    int P = fx * fy;
    size_t pitch = b->TermaBEV_pitch ? b->TermaBEV_pitch / sizeof(float) : (size_t)P;
    real* XA = (real*)calloc((size_t)n_phi * P, sizeof(real));
    real* XB = (real*)calloc((size_t)n_phi * P, sizeof(real));
    real* Dsh = (real*)calloc(P, sizeof(real));
    real* cum = (real*)calloc(P, sizeof(real));
    float dirs[24][3], base[24][3];
    const float ffx = (float)fx, ffy = (float)fy;
    for (int t = 0; t < n_theta; t++) {
        if ((double)theta[t] > 1.5707963267948966) continue;  /* forward only, DoseComp.cu:265 */
        real kA = A[t], ka = a[t], kB = B[t], kb = bb[t];
        memset(XA, 0, sizeof(real) * n_phi * P);
        memset(XB, 0, sizeof(real) * n_phi * P);
        for (int f = 0; f < n_phi; f++) {
            if (given) {
                const float* g = given + ((size_t)t_fwd * n_phi + f) * 4;
                dirs[f][0] = g[0]; dirs[f][1] = g[1]; dirs[f][2] = g[2];
            } else {
                or_cone_direction(b, theta[t], phi[f], dirs[f]);
            }
            base[f][0] = 0.5f; base[f][1] = 0.5f; base[f][2] = 0.0f;
        }
        t_fwd++;
        for (;;) {
            int s = (int)roundf(base[0][2]);
            if (s >= (int)b->long_dim) break;
            const float* Ts = terma + (size_t)s * pitch;
            const float* Rs = dens + (size_t)s * pitch;
            for (int p = 0; p < P; p++) Dsh[p] = 0;
            for (int f = 0; f < n_phi; f++) {
                real* xa = XA + (size_t)f * P;
                real* xb = XB + (size_t)f * P;
                for (int p = 0; p < P; p++) cum[p] = 0;
                int guard = 0;
                for (;;) {
                    float np[3];
                    int flag;
                    or_next_point_f(base[f], dirs[f], np, &flag);
                    for (int p = 0; p < P; p++) {
                        int ix = p % fx, iy = p / fx;
                        float btx = base[f][0] + (float)ix, bty = base[f][1] + (float)iy;
                        float ntx = np[0] + (float)ix, nty = np[1] + (float)iy;
                        float mx = (btx + ntx) * 0.5f, my = (bty + nty) * 0.5f;
                        float rx = fmodf(mx, ffx), ry = fmodf(my, ffy);
                        rx = rx < 0 ? rx + ffx : rx;
                        ry = ry < 0 ? ry + ffy : ry;
                        int cx = (int)floorf(rx), cy = (int)floorf(ry);
                        if (cx >= fx) cx = fx - 1;  /* rx rounded up to fx: last column */
                        if (cy >= fy) cy = fy - 1;
                        int mi = cx + cy * fx;
                        real T = Ts[mi], R = Rs[mi];
                        real la = xa[p], lb = xb[p];
                        double sb[3] = {btx, bty, base[f][2]}, se[3] = {ntx, nty, np[2]};
                        real pi = (real)or_calc_line_seg(sb, se, b) * R;
                        real ea = exp(-ka * pi), eb = exp(-kb * pi);
                        /* g == 1 (Q1): the local-Terma term vanishes */
                        real seg = kA / ka * la + kB / kb * lb;
                        Dsh[mi] += seg * pi;
                        cum[mi] += pi;
                        xa[p] = T * (1 - ea) + ea * la;
                        xb[p] = T * (1 - eb) + eb * lb;
                        if (floorf(btx / ffx) != floorf(ntx / ffx) || floorf(bty / ffy) != floorf(nty / ffy)) {
                            xa[p] = 0;  /* Q4: crossing a lateral edge resets the recursion */
                            xb[p] = 0;
                        }
                    }
                    base[f][0] = np[0]; base[f][1] = np[1]; base[f][2] = np[2];
                    if (flag) break;
                    if (++guard > 1000000) break;
                }
            }
            float* Ds = dose + (size_t)s * pitch;
            for (int p = 0; p < P; p++) Ds[p] = (float)((real)Ds[p] + Dsh[p] / (cum[p] + (real)EPS_FD));
        }
    }
    free(XA); free(XB); free(Dsh); free(cum);
}

/* ------------------------------------------------------------ BEV -> PVCS */
static void bev_coords(const fd2_beam_t* b, const real fwd[9], const real c[3], real cn[3]) {
    real d[3] = {c[0] - b->source[0], c[1] - b->source[1], c[2] - b->source[2]};
    real v[3];
    mv(fwd, d, v);
    real vsx = b->beamlet_size[0] * (v[1] / b->sad), vsy = b->beamlet_size[1] * (v[1] / b->sad);
    cn[0] = v[0] / vsx + (real)0.5 * b->fmap_size[0];
    cn[1] = (v[1] - b->lim_min) / b->long_spacing;
    cn[2] = v[2] / vsy + (real)0.5 * b->fmap_size[1];
}

/* d_BEV2PVCS, TermaComp.cu:124-150: texture dims (fmap_x, fmap_y, long_dim). */
void or_bev2pvcs(const fd2_beam_t* b, const float* bev, const fd2_volume_t* vol, int tm,
                 float* out) {
    real fwd[9], inv[9];
    beam_matrices(b, fwd, inv);
    int nx = vol->dim[0], ny = vol->dim[1], nz = vol->dim[2];
#pragma omp parallel for schedule(static)
    for (int z = 0; z < nz; z++)
        for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++) {
                real c[3] = {(x + (real)0.5) * vol->voxel_size[0], (y + (real)0.5) * vol->voxel_size[1],
                             (z + (real)0.5) * vol->voxel_size[2]};
                real cn[3];
                bev_coords(b, fwd, c, cn);
                out[x + (size_t)nx * (y + (size_t)ny * z)] =
                    (float)tex_linear(bev, b->fmap_size[0], b->fmap_size[1], b->long_dim, cn[0], cn[2], cn[1], tm);
            }
}

/* d_BEV2PVCS_SuperSampling, geom.cu:412-474. */
void or_bev2pvcs_ss(const fd2_beam_t* b, const float* bev, const fd2_volume_t* vol, int ss,
                    float extent, int tm, float* out) {
    real fwd[9], inv[9];
    beam_matrices(b, fwd, inv);
    int nx = vol->dim[0], ny = vol->dim[1], nz = vol->dim[2];
    real iss = (real)1 / ss;
#pragma omp parallel for schedule(static)
    for (int z = 0; z < nz; z++)
        for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++) {
                real c[3] = {(x + (real)0.5) * vol->voxel_size[0], (y + (real)0.5) * vol->voxel_size[1],
                             (z + (real)0.5) * vol->voxel_size[2]};
                real d[3] = {c[0] - b->source[0], c[1] - b->source[1], c[2] - b->source[2]}, v[3];
                mv(fwd, d, v);
                if (v[0] * v[0] + v[2] * v[2] > (real)extent * extent) continue;
                real acc = 0;
                for (int k = 0; k < ss; k++)
                    for (int j = 0; j < ss; j++)
                        for (int i = 0; i < ss; i++) {
                            real s[3] = {(x + (i + (real)0.5) * iss) * vol->voxel_size[0],
                                         (y + (j + (real)0.5) * iss) * vol->voxel_size[1],
                                         (z + (k + (real)0.5) * iss) * vol->voxel_size[2]};
                            real cn[3];
                            bev_coords(b, fwd, s, cn);
                            acc += tex_linear(bev, b->fmap_size[0], b->fmap_size[1], b->long_dim, cn[0], cn[2],
                                              cn[1], tm);
                        }
                if (acc < (real)EPS_FD) continue;
                out[x + (size_t)nx * (y + (size_t)ny * z)] = (float)(acc / ((real)ss * ss * ss));
            }
}

/* d_voxelInterp, IMRTgeom.cu:370-468: mean of ss^3 point samples of the
 * beamlet's BEV dose, samples outside the fluence map skipped, depth outside
 * [0, long_dim) reading 0.  Voxels farther than extent + half the voxel
 * diagonal from the beamlet axis are 0. */
void or_beamlet_column(const fd2_beam_t* b, const float* bev, const fd2_volume_t* vol, int ss,
                       float extent, float* row) {
    real fwd[9], inv[9];
    beam_matrices(b, fwd, inv);
    int nx = vol->dim[0], ny = vol->dim[1], nz = vol->dim[2];
    int fx = b->fmap_size[0], fy = b->fmap_size[1], L = b->long_dim;
    real vs[3] = {vol->voxel_size[0], vol->voxel_size[1], vol->voxel_size[2]};
    real hdiag = sqrt(vs[0] * vs[0] + vs[1] * vs[1] + vs[2] * vs[2]) * (real)0.5;
    real iss = (real)1 / ss;
    real icube = iss * iss * iss;
#pragma omp parallel for schedule(dynamic)
    for (int z = 0; z < nz; z++)
        for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++) {
                size_t vi = x + (size_t)nx * (y + (size_t)ny * z);
                row[vi] = 0.0f;
                real c[3] = {(x + (real)0.5) * vs[0], (y + (real)0.5) * vs[1], (z + (real)0.5) * vs[2]};
                real d[3] = {c[0] - b->source[0], c[1] - b->source[1], c[2] - b->source[2]}, v[3];
                mv(fwd, d, v);
                if (sqrt(v[0] * v[0] + v[2] * v[2]) > hdiag + extent) continue;
                real acc = 0;
                for (int kk = 0; kk < ss; kk++)
                    for (int jj = 0; jj < ss; jj++)
                        for (int ii = 0; ii < ss; ii++) {
                            real s[3] = {(x + (ii + (real)0.5) * iss) * vs[0], (y + (jj + (real)0.5) * iss) * vs[1],
                                         (z + (kk + (real)0.5) * iss) * vs[2]};
                            real cn[3];
                            bev_coords(b, fwd, s, cn);
                            if (cn[0] < 0 || cn[0] > fx || cn[2] < 0 || cn[2] > fy) continue;
                            long tx = (long)floor(cn[0]), ty = (long)floor(cn[2]), tz = (long)floor(cn[1]);
                            if (tx >= fx || ty >= fy || tz < 0 || tz >= L) continue;
                            acc += bev[tx + (size_t)fx * (ty + (size_t)fy * tz)];
                        }
                row[vi] = (float)(acc * icube);
            }
}

void or_beamlet_pipeline(const fd2_beam_t* b, const float* fluence, const float* density,
                         const fd2_volume_t* vol, int nkern, const float* energy,
                         const float* sfl, const float* mu, int n_theta, const float* theta,
                         const float* A, const float* a, const float* B, const float* bb,
                         int n_phi, const float* phi, int ss, float extent, float* row) {
    size_t n = (size_t)b->fmap_size[0] * b->fmap_size[1] * b->long_dim;
    float* T = (float*)calloc(n, sizeof(float));
    float* R = (float*)calloc(n, sizeof(float));
    float* D = (float*)calloc(n, sizeof(float));
    fd2_beam_t bc = *b;
    bc.TermaBEV_pitch = bc.DensityBEV_pitch = (uint64_t)b->fmap_size[0] * b->fmap_size[1] * sizeof(float);
    or_terma(&bc, fluence, density, vol, nkern, energy, sfl, mu, 0, T, R);
    or_cccs(&bc, T, R, n_theta, theta, A, a, B, bb, n_phi, phi, D);
    or_beamlet_column(&bc, D, vol, ss, extent, row);
    free(T); free(R); free(D);
}

/* ------------------------------------------------------------ optimizer */
static void spmv(const or_csr* M, const float* x, real* y) {
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < M->rows; r++) {
        real acc = 0;
        for (int64_t k = M->offsets[r]; k < M->offsets[r + 1]; k++) acc += (real)M->values[k] * x[M->columns[k]];
        y[r] = acc;
    }
}

/* Objective terms shared by eval_g and eval_grad (IMRTOptUtils.cu:94-155,
 * 158-222).  Optionally writes the two gradient inputs. */
static double objective(const or_problem* p, const float* x, float* g1in, float* g2in) {
    int64_t nv = p->n_ptv + p->n_oar;
    real* Ax = (real*)malloc(sizeof(real) * (nv ? nv : 1));
    real* Dx = (real*)malloc(sizeof(real) * (p->D.rows ? p->D.rows : 1));
    spmv(&p->A, x, Ax);
    spmv(&p->D, x, Dx);
    double s1 = 0, s2 = 0, s3 = 0, s4 = 0, s5 = 0;
    for (int64_t i = 0; i < nv; i++) {
        real ax = (real)(float)Ax[i];
        real pr2 = ax - p->max_dose[i] > 0 ? ax - p->max_dose[i] : 0;  /* d_calc_prox2 */
        s2 += fabs((double)p->max_weights[i] * pr2 * pr2);
        real v1;
        if (i < p->n_ptv) {
            real pr1 = ax - p->min_dose[i] < 0 ? ax - p->min_dose[i] : 0;  /* d_calc_prox1 */
            s1 += fabs((double)p->min_weights[i] * pr1 * pr1);
            v1 = p->min_weights[i] * pr1;
        } else {
            real t3 = ax;  /* term3 */
            s3 += fabs((double)p->oar_weights[i - p->n_ptv] * t3 * t3);
            v1 = p->oar_weights[i - p->n_ptv] * t3;
        }
        if (g1in) g1in[i] = (float)(v1 + p->max_weights[i] * pr2);  /* d_calc_grad_term1_input */
    }
    for (int64_t i = 0; i < p->D.rows; i++) {
        real t4 = (real)(float)Dx[i];
        real m = fabs(t4) - p->gamma;
        m = m > 0 ? m : 0;
        real pr4 = m * (real)((t4 > 0) - (t4 < 0));  /* d_prox1Norm */
        s4 += fabs(pr4);
        s5 += (pr4 - t4) * (pr4 - t4);
        if (g2in) g2in[i] = (float)((t4 - pr4) * ((real)p->eta / p->gamma));  /* d_calc_grad_term2_input */
    }
    free(Ax); free(Dx);
    return 0.5 * (s1 + s2 + s3) + (double)p->eta * (s4 + 0.5 / (double)p->gamma * s5);
}

double or_eval_g(const or_problem* p, const float* x) { return objective(p, x, NULL, NULL); }

double or_eval_grad(const or_problem* p, const float* x, float* grad) {
    int64_t nv = p->n_ptv + p->n_oar;
    float* g1 = (float*)malloc(sizeof(float) * (nv ? nv : 1));
    float* g2 = (float*)malloc(sizeof(float) * (p->D.rows ? p->D.rows : 1));
    double g = objective(p, x, g1, g2);
    int64_t n = p->AT.rows;
    real* o1 = (real*)malloc(sizeof(real) * (n ? n : 1));
    real* o2 = (real*)malloc(sizeof(real) * (n ? n : 1));
    spmv(&p->AT, g1, o1);
    spmv(&p->DT, g2, o2);
    for (int64_t i = 0; i < n; i++) grad[i] = (float)((real)(float)o1[i] + (real)(float)o2[i]);  /* d_elementWiseAdd */
    free(g1); free(g2); free(o1); free(o2);
    return g;
}

#define TWO_OVER_ROOT3 1.1547005383792517
#define THREE_QUARTERS_ROOT3 1.299038105676658
#define PI_OVER_TWO 1.5707963267948966
#define TWO_TIMES_ROOT6_OVER_NINE 0.5443310539518174

/* d_proxL2Onehalf_calc_tHat, IMRTOptimize_var1.cu:544-570: closed-form
 * minimiser scale of tau*||x||^(1/2) + ||x - g||^2/2 along g (the 2021 QL
 * formula), with the reference's zero-norm guard (nrm2 <= 1e-4 -> 1008611). */
double or_that(double nrm2, double tau) {
    double n34 = 1008611.0;
    if (nrm2 > (double)EPS_FD) n34 = pow(nrm2, -0.75);
    double alpha = tau * n34;
    if (alpha > TWO_TIMES_ROOT6_OVER_NINE) return 0.0;
    double s = sin((acos(alpha * THREE_QUARTERS_ROOT3) + PI_OVER_TWO) / 3.0) * TWO_OVER_ROOT3;
    return s * s;
}

void or_prox_l2onehalf(int64_t ng, const int64_t* go, const float* g0, const float* tau, float* prox,
                       float* nrmnew) {
    for (int64_t r = 0; r < ng; r++) {
        double n2 = 0;
        for (int64_t k = go[r]; k < go[r + 1]; k++) n2 += (double)g0[k] * g0[k];
        double th = or_that((double)(float)n2, tau[r]);
        double m2 = 0;
        for (int64_t k = go[r]; k < go[r + 1]; k++) {
            prox[k] = (float)(th * g0[k]);
            m2 += (double)prox[k] * prox[k];
        }
        nrmnew[r] = (float)sqrt((double)(float)m2);
    }
}

static double dotf(int64_t n, const float* a, const float* b) {
    double s = 0;
    for (int64_t i = 0; i < n; i++) s += (double)a[i] * b[i];
    return s;
}

int or_boo_l2onehalf(const or_problem* p, int64_t ng, const int64_t* go, float* w, int show,
                     int change_trigger, int iters_global, const int* prune, int n_prune,
                     int want, or_opt_state* st) {
    int64_t n = p->AT.rows;
    float *x = malloc(4 * n), *y = malloc(4 * n), *v = malloc(4 * n), *g = malloc(4 * n);
    float *in = malloc(4 * n), *tw = malloc(4 * ng);
    int iters_local = iters_global;
    for (int i = 0; i < n_prune; i++)
        if (prune[i] > st->k_global) { iters_local = prune[i] - st->k_global; break; }
    float t = st->tkm1, theta = 1.0f;
    double gx = 0;
    st->stop = 0;
    st->trials = 0;
    (void)show;
    int k_local = 0;
    for (; st->k_global < iters_global && k_local < iters_local; st->k_global++, k_local++) {
        if (st->k_global < 50 || st->k_global % 5 == 0) t /= 0.5f;
        for (;;) {
            st->trials++;
            if (st->k_global > 1) {
                float aa = st->tkm1, bb = t * st->theta_km1 * st->theta_km1, cc = -bb;
                theta = (-bb + sqrtf(bb * bb - 4 * aa * cc)) / (2 * aa);
                for (int64_t i = 0; i < n; i++) y[i] = (1.0f - theta) * st->xkm1[i] + theta * st->vkm1[i];
            } else {
                theta = 1.0f;
                memcpy(y, st->xkm1, 4 * n);
            }
            double gy = or_eval_grad(p, y, g);
            for (int64_t i = 0; i < n; i++) {
                float val = 1.0f * y[i] + (-t) * g[i];
                in[i] = val > 0.0f ? val : 0.0f;
            }
            for (int64_t r = 0; r < ng; r++) tw[r] = w[r] * t;
            or_prox_l2onehalf(ng, go, in, tw, x, st->nrm);
            gx = or_eval_g(p, x);
            double dxy = 0, nxy = 0;
            for (int64_t i = 0; i < n; i++) {
                float dlt = 1.0f * x[i] + (-1.0f) * y[i];
                dxy += (double)g[i] * dlt;
                nxy += (double)dlt * dlt;
            }
            double rhs = gy + dxy + (0.5 / t) * nxy;
            if (gx <= rhs) break;
            t *= 0.5f;
        }
        float iot = 1.0f / theta;
        for (int64_t i = 0; i < n; i++) v[i] = iot * x[i] + (1.0f - iot) * st->xkm1[i];
        st->theta_km1 = theta;
        st->tkm1 = t;
        memcpy(st->xkm1, x, 4 * n);
        memcpy(st->vkm1, v, 4 * n);
        double cost = 0;
        float active = 0;
        for (int64_t r = 0; r < ng; r++) {
            cost += (double)w[r] * sqrt((double)st->nrm[r]);
            active += st->nrm[r] > 1e-4f;
        }
        st->loss[st->k_global] = (float)(cost + gx);
        st->num_active = active;
        if (active - EPS_FD <= want) { st->stop = 1; break; }
        if ((st->k_global + 1) % change_trigger == 0) {
            float sc = 1.0f;
            if (active >= 2 * want) sc = 2.0f;
            else if (active >= 1.5f * want) sc = 1.5f;
            else if (active >= 1.05f * want) sc = 1.2f;
            else if (active < want) sc = 0.3333f;
            if (sc != 1.0f) for (int64_t r = 0; r < ng; r++) w[r] *= sc;
        }
    }
    if (st->k_global == iters_global) st->stop = 1;
    (void)dotf;
    free(x); free(y); free(v); free(g); free(in); free(tw);
    return 0;
}

int or_polish(const or_problem* p, int iters_global, int iters_local, or_opt_state* st) {
    int64_t n = p->AT.rows;
    float *x = malloc(4 * n), *y = malloc(4 * n), *v = malloc(4 * n), *g = malloc(4 * n);
    float t = st->tkm1, theta = 1.0f;
    st->trials = 0;
    int k_local = 0;
    for (; st->k_global < iters_global && k_local < iters_local; st->k_global++, k_local++) {
        if (st->k_global < 50 || st->k_global % 5 == 0) t /= 0.5f;
        double gx;
        for (;;) {
            st->trials++;
            if (st->k_global > 1) {
                float aa = st->tkm1, bb = t * st->theta_km1 * st->theta_km1, cc = -bb;
                theta = (-bb + sqrtf(bb * bb - 4 * aa * cc)) / (2 * aa);
                for (int64_t i = 0; i < n; i++) y[i] = (1.0f - theta) * st->xkm1[i] + theta * st->vkm1[i];
            } else {
                theta = 1.0f;
                memcpy(y, st->xkm1, 4 * n);
            }
            double gy = or_eval_grad(p, y, g);
            for (int64_t i = 0; i < n; i++) {
                float val = 1.0f * y[i] + (-t) * g[i];
                x[i] = val > 0.0f ? val : 0.0f;
            }
            gx = or_eval_g(p, x);
            double dxy = 0, nxy = 0;
            for (int64_t i = 0; i < n; i++) {
                float dlt = 1.0f * x[i] + (-1.0f) * y[i];
                dxy += (double)g[i] * dlt;
                nxy += (double)dlt * dlt;
            }
            double rhs = gy + dxy + (0.5 / t) * nxy;
            if (gx <= rhs) break;
            t *= 0.5f;
        }
        float iot = 1.0f / theta;
        for (int64_t i = 0; i < n; i++) v[i] = iot * x[i] + (1.0f - iot) * st->xkm1[i];
        st->theta_km1 = theta;
        st->tkm1 = t;
        memcpy(st->xkm1, x, 4 * n);
        memcpy(st->vkm1, v, 4 * n);
        st->loss[st->k_global] = (float)gx;
    }
    free(x); free(y); free(v); free(g);
    return 0;
}

void or_beam_weights_init(int64_t nb, const or_csr* Ab, int64_t n_ptv, float* out) {
    for (int64_t b = 0; b < nb; b++) {
        const or_csr* M = &Ab[b];
        double s = 0;
        for (int64_t r = 0; r < n_ptv && r < M->rows; r++)
            for (int64_t k = M->offsets[r]; k < M->offsets[r + 1]; k++) s += M->values[k];
        out[b] = sqrtf((float)s / (float)(n_ptv * M->cols));
    }
    float mx = 0.0f;
    for (int64_t b = 0; b < nb; b++) mx = out[b] > mx ? out[b] : mx;
    for (int64_t b = 0; b < nb; b++) {
        out[b] /= mx;
        if (out[b] < 0.1f) out[b] = 0.1f;
    }
}

void or_fluence_grad(int n, const uint8_t* act, int64_t* rows, int64_t* nnz, int64_t* off,
                     int64_t* col, float* val) {
    /* column index of each active pixel (filterConstruction, IMRTEigenLoad.cpp:437-459) */
    int64_t* cidx = (int64_t*)malloc(sizeof(int64_t) * n * n);
    int64_t na = 0;
    for (int p = 0; p < n * n; p++) cidx[p] = act[p] ? na++ : -1;
    int64_t r = 0, z = 0;
    off[0] = 0;
    /* Dx rows: kron(I, Dxy), row y*n + x joins pixels (x, x+1) of row y; kept
     * only when both ends are active (sum ~ 0 and |.|-sum > 0). */
    for (int pass = 0; pass < 2; pass++) {
        for (int q = 0; q < n * n; q++) {
            int p0, p1;
            if (pass == 0) {
                int y = q / n, x = q % n;
                if (x >= n - 1) continue;
                p0 = y * n + x; p1 = y * n + x + 1;
            } else {
                int yy = q / n, x = q % n;  /* kron(Dxy, I): row yy*n + x joins (x,yy),(x,yy+1) */
                if (yy >= n - 1) continue;
                p0 = yy * n + x; p1 = (yy + 1) * n + x;
            }
            if (cidx[p0] < 0 || cidx[p1] < 0) continue;
            col[z] = cidx[p0]; val[z] = -1.0f; z++;
            col[z] = cidx[p1]; val[z] = 1.0f; z++;
            r++;
            off[r] = z;
        }
    }
    *rows = r;
    *nnz = z;
    free(cidx);
}
