/*
 * vamoracle.c -- CPU restatement of the VAMToolbox projection hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: tests/, the
 * smoke check and bench.py's CPU-baseline leg call it as the checker and as
 * the timed CPU baseline.  The product path (vamtoolbox_b200) never links or
 * calls it.
 *
 * Precision follows the reference exactly where it matters:
 *   - parallel beam: float64 throughout, coordinates and interpolation in the
 *     operation order of skimage.transform.warp (order 1, constant mode, cval
 *     0) and np.interp, as called by
 *     vamtoolbox/projector/Projector3DParallel.py:113-207;
 *   - ray tracer: float32 ray state and float64 field sampling, as in
 *     vamtoolbox/projector/pyTorchRayTrace.py:738-775 with fields built from
 *     float64 numpy coordinates (RayState default dtype, :1445-1458).
 * Compiled with -ffp-contract=off so no multiply-add is fused (the reference's
 * numpy / Cython builds target baseline x86-64 without FMA).
 *
 * Parity pins: tests/golden/*.npz, generated by running the reference's own
 * Python code (tests/golden/make_golden.py); the one third-party routine the
 * reference calls that is absent here (skimage.transform.warp, scikit-image,
 * version unpinned in conda/meta.yaml:32) is restated from its documented
 * behaviour: inverse map (col, row, 1) @ M^T, bilinear with floor/ceil
 * neighbours, zero outside.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ---------------------------------------------------------------------- */
/* parallel beam                                                          */
/* ---------------------------------------------------------------------- */

/* numpy: np.cos(np.deg2rad(a)), deg2rad(a) = a * (pi/180) */
static void angle_tables(const double* ang, int nA, double* c, double* s) {
    for (int i = 0; i < nA; ++i) {
        double r = ang[i] * (M_PI / 180.0);
        c[i] = cos(r);
        s[i] = sin(r);
    }
}

/* Projector3DParallel.py:137-143: R = [[c, s, -C(c+s-1)], [-s, c, -C(c-s-1)], [0,0,1]] */
static void warp_matrix(double c, double s, int C, double* m) {
    m[0] = c;
    m[1] = s;
    m[2] = -(double)C * ((c + s) - 1.0);
    m[3] = -s;
    m[4] = c;
    m[5] = -(double)C * ((c - s) - 1.0);
}

static inline double pix(const double* img, int rows, int cols, long r, long c, int nZ, int z) {
    if (r < 0 || r >= rows || c < 0 || c >= cols) return 0.0;
    return img[((size_t)r * cols + c) * nZ + z];
}

/* skimage bilinear sample of slice z at (r, c): floor/ceil corners, zero outside */
static inline double bilinear(const double* img, int rows, int cols, int nZ, int z, double r, double c) {
    long minr = (long)floor(r), minc = (long)floor(c);
    long maxr = (long)ceil(r), maxc = (long)ceil(c);
    double dr = r - (double)minr, dc = c - (double)minc;
    double tl = pix(img, rows, cols, minr, minc, nZ, z);
    double tr = pix(img, rows, cols, minr, maxc, nZ, z);
    double bl = pix(img, rows, cols, maxr, minc, nZ, z);
    double br = pix(img, rows, cols, maxr, maxc, nZ, z);
    double top = (1.0 - dc) * tl + dc * tr;
    double bottom = (1.0 - dc) * bl + dc * br;
    return (1.0 - dr) * top + dr * bottom;
}

/* Per-sample absorption weight of the RAY mode at detector offset t, depth s. */
static inline double ray_abs_weight(double t, double s, double alpha, double R) {
    if (fabs(t) > R) return 0.0;
    double s_entry = -sqrt(R * R - t * t);
    double d = s - s_entry;
    return d > 0.0 ? exp(-alpha * d) : 1.0;
}

/*
 * R1 forward.  x: [nY][nX][nZ], b: [nY][nA][nZ].  occ (optional): occlusion
 * sinogram [nY][nA][nZ] with NaN for "no occluder", occ_flag [nA][nZ].
 * abs_mode: 0 none, 1 mask (x multiplied by mask[nY][nX] first), 2 ray.
 */
void orc_parallel_forward(const double* x, int nY, int nX, int nZ, const double* ang, int nA,
                          const double* occ, const uint8_t* occ_flag, int abs_mode,
                          const double* mask, double alpha, double R, double* b) {
    int C = nY / 2;
    double* cs = (double*)malloc(sizeof(double) * 2 * nA);
    angle_tables(ang, nA, cs, cs + nA);
    const double* xin = x;
    double* xm = NULL;
    if (abs_mode == 1) {
        xm = (double*)malloc(sizeof(double) * (size_t)nY * nX * nZ);
        for (size_t p = 0; p < (size_t)nY * nX; ++p)
            for (int z = 0; z < nZ; ++z) xm[p * nZ + z] = mask[p] * x[p * nZ + z];
        xin = xm;
    }
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
    for (int z = 0; z < nZ; ++z) {
        for (int i = 0; i < nA; ++i) {
            double m[6];
            warp_matrix(cs[i], cs[nA + i], C, m);
            int use_occ = occ && occ_flag[(size_t)i * nZ + z];
            for (int j = 0; j < nX; ++j) {
                double acc = 0.0;
                double occv = use_occ ? occ[((size_t)j * nA + i) * nZ + z] : NAN;
                for (int k = 0; k < nY; ++k) {
                    /* _transform_affine: x_ = H0*x + H1*y + H2 with x = col j, y = row k */
                    double cin = (m[0] * (double)j + m[1] * (double)k) + m[2];
                    double rin = (m[3] * (double)j + m[4] * (double)k) + m[5];
                    double v = bilinear(xin, nY, nX, nZ, z, rin, cin);
                    if (use_occ && ((double)(k - C) > occv)) v = 0.0;
                    if (abs_mode == 2) v *= ray_abs_weight((double)(j - C), (double)(k - C), alpha, R);
                    acc += v;
                }
                b[((size_t)j * nA + i) * nZ + z] = acc;
            }
        }
    }
    free(xm);
    free(cs);
}

/*
 * Exact transpose of orc_parallel_forward (scatter form): every sample's four
 * skimage taps receive b * tap weight * sample factor.
 */
void orc_parallel_adjoint(const double* b, int nY, int nX, int nZ, const double* ang, int nA,
                          const double* occ, const uint8_t* occ_flag, int abs_mode,
                          const double* mask, double alpha, double R, double* x) {
    int C = nY / 2;
    double* cs = (double*)malloc(sizeof(double) * 2 * nA);
    angle_tables(ang, nA, cs, cs + nA);
    memset(x, 0, sizeof(double) * (size_t)nY * nX * nZ);
#pragma omp parallel for schedule(dynamic, 1)
    for (int z = 0; z < nZ; ++z) {
        for (int i = 0; i < nA; ++i) {
            double m[6];
            warp_matrix(cs[i], cs[nA + i], C, m);
            int use_occ = occ && occ_flag[(size_t)i * nZ + z];
            for (int j = 0; j < nX; ++j) {
                double bv = b[((size_t)j * nA + i) * nZ + z];
                double occv = use_occ ? occ[((size_t)j * nA + i) * nZ + z] : NAN;
                for (int k = 0; k < nY; ++k) {
                    if (use_occ && ((double)(k - C) > occv)) continue;
                    double f = bv;
                    if (abs_mode == 2) f *= ray_abs_weight((double)(j - C), (double)(k - C), alpha, R);
                    double cin = (m[0] * (double)j + m[1] * (double)k) + m[2];
                    double rin = (m[3] * (double)j + m[4] * (double)k) + m[5];
                    long minr = (long)floor(rin), minc = (long)floor(cin);
                    long maxr = (long)ceil(rin), maxc = (long)ceil(cin);
                    double dr = rin - (double)minr, dc = cin - (double)minc;
                    long rr[4] = {minr, minr, maxr, maxr};
                    long cc[4] = {minc, maxc, minc, maxc};
                    double ww[4] = {(1.0 - dr) * (1.0 - dc), (1.0 - dr) * dc, dr * (1.0 - dc), dr * dc};
                    for (int t = 0; t < 4; ++t) {
                        if (rr[t] < 0 || rr[t] >= nY || cc[t] < 0 || cc[t] >= nX) continue;
                        x[((size_t)rr[t] * nX + cc[t]) * nZ + z] += ww[t] * f;
                    }
                }
            }
        }
    }
    if (abs_mode == 1) {
        for (size_t p = 0; p < (size_t)nY * nX; ++p)
            for (int z = 0; z < nZ; ++z) x[p * nZ + z] *= mask[p];
    }
    free(cs);
}

/* np.interp(t, xp = arange(n) - n//2, fp, left, right) for unit-spaced integer xp */
static inline double np_interp_unit(double t, const double* fp, size_t stride, int n, int x0,
                                    double left, double right) {
    double xlo = (double)x0, xhi = (double)(x0 + n - 1);
    if (isnan(t)) return t;
    if (t < xlo) return left;
    if (t > xhi) return right;
    if (t == xhi) return fp[(size_t)(n - 1) * stride];
    /* bin j with xp[j] <= t < xp[j+1]; floor(t) is exact, floor(t - xp[0]) is not */
    long j = (long)floor(t) - (long)x0;
    double xj = xlo + (double)j;
    double yj = fp[(size_t)j * stride];
    if (xj == t) return yj;
    double yj1 = fp[(size_t)(j + 1) * stride];
    double slope = (yj1 - yj) / 1.0;
    double res = slope * (t - xj) + yj;
    if (isnan(res)) {
        res = slope * (t - (xj + 1.0)) + yj1;
        if (isnan(res) && yj == yj1) res = yj;
    }
    return res;
}

/* numpy linspace(-1, 1, n)[i] */
static inline double lin_m1_1(int i, int n) {
    if (n == 1) return -1.0;
    if (i == n - 1) return 1.0;
    double step = 2.0 / (double)(n - 1);
    return (double)i * step + -1.0;
}

/* vamtoolbox/util/data.py:14-40: zero where lin[i]^2 + lin[j]^2 > 1 */
int orc_circle_inside(int i, int j, int nY, int nX) {
    double a = lin_m1_1(i, nY), c = lin_m1_1(j, nX);
    return !((a * a + c * c) > 1.0);
}

/*
 * R2 reference-parity backprojection (Projector3DParallel.py:158-207).
 * abs_mode 1 multiplies by mask before the clip (Projector3DParallel.py:51-54);
 * abs_mode 2 weights each (pixel, angle) by the ray absorption factor.
 */
void orc_parallel_backward_ref(const double* b, int nY, int nX, int nZ, const double* ang, int nA,
                               const double* occ, int abs_mode, const double* mask, double alpha,
                               double R, double* x) {
    int C = nY / 2;
    double* cs = (double*)malloc(sizeof(double) * 2 * nA);
    angle_tables(ang, nA, cs, cs + nA);
#pragma omp parallel for collapse(2) schedule(dynamic, 4)
    for (int z = 0; z < nZ; ++z) {
        for (int i = 0; i < nY; ++i) {
            for (int j = 0; j < nX; ++j) {
                double X = (double)(j - C), Y = (double)(i - C);
                double acc = 0.0;
                for (int a = 0; a < nA; ++a) {
                    double c = cs[a], s = cs[nA + a];
                    double t = X * c - Y * s;
                    double sv = X * s + Y * c;
                    double v = np_interp_unit(t, b + (size_t)a * nZ + z, (size_t)nA * nZ, nY, -C, 0.0, 0.0);
                    if (occ) {
                        double o = np_interp_unit(t, occ + (size_t)a * nZ + z, (size_t)nA * nZ, nY, -C, NAN, NAN);
                        if (sv > floor(o)) v = 0.0;
                    }
                    if (abs_mode == 2) v *= ray_abs_weight(t, sv, alpha, R);
                    acc += v;
                }
                if (abs_mode == 1) acc = mask[(size_t)i * nX + j] * acc;
                if (!orc_circle_inside(i, j, nY, nX)) acc = 0.0;
                x[((size_t)i * nX + j) * nZ + z] = acc;
            }
        }
    }
    free(cs);
}

/*
 * Occlusion sinogram (Projector3DParallel.py:77-111): min over rows k of
 * (k - C) where warp(insert) > 0, NaN if none.  occ_flag[a][z] reproduces the
 * forward's gate `count_nonzero(occ) - sum(isnan(occ)) != 0` (:149).
 */
void orc_occlusion_sinogram(const double* insert, int nY, int nX, int nZ, const double* ang, int nA,
                            double* occ, uint8_t* occ_flag) {
    int C = nY / 2;
    double* cs = (double*)malloc(sizeof(double) * 2 * nA);
    angle_tables(ang, nA, cs, cs + nA);
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
    for (int z = 0; z < nZ; ++z) {
        for (int i = 0; i < nA; ++i) {
            double m[6];
            warp_matrix(cs[i], cs[nA + i], C, m);
            int finite_nonzero = 0;
            for (int j = 0; j < nX; ++j) {
                double best = NAN;
                for (int k = 0; k < nY; ++k) {
                    double cin = (m[0] * (double)j + m[1] * (double)k) + m[2];
                    double rin = (m[3] * (double)j + m[4] * (double)k) + m[5];
                    if (bilinear(insert, nY, nX, nZ, z, rin, cin) > 0.0) {
                        best = (double)(k - C);
                        break; /* rows are scanned in increasing y */
                    }
                }
                occ[((size_t)j * nA + i) * nZ + z] = best;
                if (!isnan(best) && best != 0.0) finite_nonzero = 1;
            }
            occ_flag[(size_t)i * nZ + z] = (uint8_t)finite_nonzero;
        }
    }
    free(cs);
}

/* ---------------------------------------------------------------------- */
/* curved-ray tracer                                                      */
/* ---------------------------------------------------------------------- */

typedef struct {
    int nx, ny, nz;
    double span[3];      /* grid_span = max - min per axis                       */
    double xmax[3];      /* xv_yv_zv_max                                         */
    double xmin[3];
    double voxel[3];     /* voxel size (inf for z in 2D)                         */
    double norm[3];      /* position_normalization_factor = 2/span (0 for 2D z) */
    float h32;           /* step size as the float32 the reference multiplies by */
    double h_idx;        /* step_size / voxel_x                                  */
    int max_steps, check_every, twod;
    /* index */
    int n_kind;          /* 0 homogeneous (float n_sur), 1 grid (double)         */
    float n_sur;
    const double* n_grid;    /* [nx][ny][nz]      */
    const double* g_grid;    /* [nx][ny][nz][3]   */
    /* attenuation */
    int a_kind;          /* 0 zero, 1 cylinder, 2 ball, 3 grid                    */
    float a_val, a_R;
    const double* a_grid;
    const double* absorb;    /* alpha_abs at grid points [nx][ny][nz] */
} orc_ray_cfg;

/* torch grid_sample, 5-D input, bilinear, align_corners=True; border clamps the
 * unnormalised coordinate into [0, size-1], zeros padding skips outside corners. */
static double grid_sample3(const double* f, int nch, int ch, const orc_ray_cfg* g, const float* xp,
                           int border) {
    double u[3], ix[3];
    int size[3] = {g->nx, g->ny, g->nz};
    for (int d = 0; d < 3; ++d) {
        u[d] = (double)xp[d] * g->norm[d];
        ix[d] = ((u[d] + 1.0) / 2.0) * (double)(size[d] - 1);
        if (border) ix[d] = fmin((double)(size[d] - 1), fmax(ix[d], 0.0));
    }
    long x0 = (long)floor(ix[0]), y0 = (long)floor(ix[1]), z0 = (long)floor(ix[2]);
    double wx1 = ix[0] - (double)x0, wx0 = (double)(x0 + 1) - ix[0];
    double wy1 = ix[1] - (double)y0, wy0 = (double)(y0 + 1) - ix[1];
    double wz1 = ix[2] - (double)z0, wz0 = (double)(z0 + 1) - ix[2];
    double out = 0.0;
    for (int cz = 0; cz < 2; ++cz)
        for (int cy = 0; cy < 2; ++cy)
            for (int cx = 0; cx < 2; ++cx) {
                long X = x0 + cx, Y = y0 + cy, Z = z0 + cz;
                if (X < 0 || X >= g->nx || Y < 0 || Y >= g->ny || Z < 0 || Z >= g->nz) continue;
                double w = (cx ? wx1 : wx0) * (cy ? wy1 : wy0) * (cz ? wz1 : wz0);
                out += f[(((size_t)X * g->ny + Y) * g->nz + Z) * nch + ch] * w;
            }
    return out;
}

/* attenuation coefficient at x_i: analytic kinds are float32 in the reference */
static double alpha_att(const orc_ray_cfg* g, const float* x, int* is_float) {
    *is_float = 0;
    if (g->a_kind == 0) { *is_float = 1; return 0.0; }
    if (g->a_kind == 1 || g->a_kind == 2) {
        float r2 = x[0] * x[0] + x[1] * x[1];
        if (g->a_kind == 2) r2 += x[2] * x[2];
        float r = sqrtf(r2);
        *is_float = 1;
        return (r < g->a_R) ? (double)g->a_val : 0.0;
    }
    return grid_sample3(g->a_grid, 1, 0, g, x, 0);
}

/*
 * Trace every ray (symplectic Euler, physical path length) until the step
 * cap, exiting rays per the 10-step exit check.  mode 0: integrate f into
 * out_g[ray]; mode 1: deposit g[ray] into out_dose (double grid).
 * Returns the number of rays still active at the cap.
 */
long orc_ray_trace(const orc_ray_cfg* g, const float* x0, const float* v0, float energy0, long nrays,
                   int mode, const double* f, const float* gin, float* out_g, double* out_dose) {
    long still_active = 0;
    size_t ngrid = (size_t)g->nx * g->ny * g->nz;
    double* fa = NULL;
    if (mode == 0) {
        fa = (double*)malloc(sizeof(double) * ngrid);
        for (size_t v = 0; v < ngrid; ++v) fa[v] = f[v] * g->absorb[v];
    }
    int nthreads = 1;
#ifdef _OPENMP
    nthreads = omp_get_max_threads();
#endif
    double* dose_t = NULL;
    if (mode == 1) {
        dose_t = (double*)calloc((size_t)nthreads * ngrid, sizeof(double));
    }
    int ncorner = g->twod ? 4 : 8;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : still_active)
    for (long r = 0; r < nrays; ++r) {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double* dose = mode == 1 ? dose_t + (size_t)tid * ngrid : NULL;
        float xi[3], xp[3], vi[3], vp[3];
        for (int d = 0; d < 3; ++d) {
            xi[d] = xp[d] = x0[r * 3 + d];
            vi[d] = vp[d] = v0[r * 3 + d];
        }
        float s = 0.f, att = 0.f, integral = 0.f;
        float E0 = mode == 1 ? gin[r] : energy0;
        float E = E0;
        int active = 1;
        for (int step = 0; step < g->max_steps; ++step) {
            if (active) {
                for (int d = 0; d < 3; ++d) { xi[d] = xp[d]; vi[d] = vp[d]; }
                /* v_ip1 = v_i + grad_n(x_i).float() * h */
                for (int d = 0; d < 3; ++d) {
                    float gd;
                    if (g->n_kind == 0) gd = 0.f;
                    else gd = (float)grid_sample3(g->g_grid, 3, d, g, xi, 1);
                    vp[d] = vi[d] + gd * g->h32;
                }
                /* dx = (v_ip1 / n(x_i)).float() * h */
                float dx[3];
                if (g->n_kind == 0) {
                    for (int d = 0; d < 3; ++d) dx[d] = (vp[d] / g->n_sur) * g->h32;
                } else {
                    double n = grid_sample3(g->n_grid, 1, 0, g, xi, 1);
                    for (int d = 0; d < 3; ++d) dx[d] = ((float)((double)vp[d] / n)) * g->h32;
                }
                for (int d = 0; d < 3; ++d) xp[d] = xi[d] + dx[d];
                float ds = (float)sqrt((double)dx[0] * dx[0] + (double)dx[1] * dx[1] + (double)dx[2] * dx[2]);
                s += ds;
                int af;
                double a = alpha_att(g, xi, &af);
                if (af) att = att + (float)a * ds;
                else att = (float)((double)att + a * (double)ds);
                E = E0 * expf(-att);
                /* deposit / integrate at x_ip1 */
                double idx[3];
                long lo[3], hi[3];
                for (int d = 0; d < 3; ++d) {
                    idx[d] = ((double)xp[d] - (-g->span[d] / 2.0)) * (1.0 / g->voxel[d]);
                    lo[d] = (long)floor(idx[d]);
                    hi[d] = (long)ceil(idx[d]);
                }
                for (int cn = 0; cn < ncorner; ++cn) {
                    long X = (cn & 1) ? hi[0] : lo[0];
                    long Y = (cn & 2) ? hi[1] : lo[1];
                    long Z = (cn & 4) ? hi[2] : lo[2];
                    if (X < 0 || X >= g->nx || Y < 0 || Y >= g->ny || Z < 0 || Z >= g->nz) continue;
                    double coef = (1.0 - fabs(idx[0] - (double)X)) * (1.0 - fabs(idx[1] - (double)Y));
                    coef = coef * (1.0 - fabs(idx[2] - (double)Z));
                    double en = (g->h_idx * coef) * (double)E;
                    size_t v = ((size_t)X * g->ny + Y) * g->nz + Z;
                    if (mode == 0) integral = (float)((double)integral + fa[v] * en);
                    else dose[v] += en;
                }
            }
            if (step % g->check_every == 0 && active) {
                for (int d = 0; d < 3; ++d) {
                    int pos = ((double)xp[d] > g->xmax[d] + g->voxel[d]) && (vp[d] > 0.f);
                    int neg = ((double)xp[d] < g->xmin[d] - g->voxel[d]) && (vp[d] < 0.f);
                    if (pos || neg) active = 0;
                }
            }
        }
        if (active) still_active += 1;
        if (mode == 0) out_g[r] = integral;
    }
    if (mode == 1) {
        for (size_t v = 0; v < ngrid; ++v) {
            double acc = 0.0;
            for (int t = 0; t < nthreads; ++t) acc += dose_t[(size_t)t * ngrid + v];
            out_dose[v] = acc * g->absorb[v];
        }
        free(dose_t);
    }
    free(fa);
    return still_active;
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
