/*
 * EDGE oracle: a plain-C (float32, OpenMP) restatement of the reference's
 * per-step kernels.  TEST INFRASTRUCTURE ONLY: it is the checker for the CUDA
 * library and the timed CPU baseline; nothing in the product links it.
 *
 * Parity is pinned by the .npz fixtures in tests/golden, which were produced by executing the
 * reference's own Python sources (numpy emulation of Taichi, see
 * tests/golden/make_golden.py).  Every function cites the reference lines it
 * restates; arithmetic order follows the reference expressions so that float32
 * results agree to a few ulps (compile with -ffp-contract=off).
 *
 * Layout (row-major, z fastest, like Taichi's to_numpy()):
 *   scalar field  f[(i*ny + j)*nz + k]
 *   vec3 field    f[((i*ny + j)*nz + k)*3 + c]
 *   vec4 dye      f[((i*ny + j)*nz + k)*4 + c]
 * Face grids of an (nx,ny,nz) cell grid: u_x (nx+1,ny,nz), u_y (nx,ny+1,nz),
 * u_z (nx,ny,nz+1).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define EXPORT __attribute__((visibility("default")))

/* taichi_utils.py:3 — eps = 1e-6; the clamp bounds dim-2-eps / dim-1-eps are
 * Python constants folded in double and narrowed to float32 (default_fp). */
#define REF_EPS 1e-6

/* loops over fewer elements than this run on one thread (tiny multigrid
 * levels would otherwise pay an OpenMP fork/join per half sweep) */
#define OMP_MIN 32768

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline float fminr(float a, float b) { return a < b ? a : b; }
static inline float fmaxr(float a, float b) { return a > b ? a : b; }
static inline size_t ix3(int i, int j, int k, int ny, int nz) { return ((size_t)i * ny + j) * nz + k; }

typedef struct { const float *p; int n0, n1, n2; } sf_t; /* scalar field view */

/* taichi_utils.py:62-67 sample(): integer clamp to the field shape */
static inline float samp(sf_t f, int i, int j, int k) {
    i = clampi(i, 0, f.n0 - 1);
    j = clampi(j, 0, f.n1 - 1);
    k = clampi(k, 0, f.n2 - 1);
    return f.p[ix3(i, j, k, f.n1, f.n2)];
}
static inline const float *samp_v(const float *f, int n0, int n1, int n2, int nc, int i, int j, int k) {
    i = clampi(i, 0, n0 - 1);
    j = clampi(j, 0, n1 - 1);
    k = clampi(k, 0, n2 - 1);
    return f + ix3(i, j, k, n1, n2) * nc;
}

/* ------------------------------------------------------------------------ */
/* B-spline and trilinear kernels                                            */
/* ------------------------------------------------------------------------ */
/* taichi_utils.py:230-238 N_2 */
static inline float N2(float x) {
    float r = 0.0f, a = fabsf(x);
    if (a < 0.5f) r = 0.75f - a * a;
    else if (a < 1.5f) { float t = 1.5f - a; r = 0.5f * (t * t); }
    return r;
}
/* taichi_utils.py:241-251 dN_2 */
static inline float dN2(float x) {
    float r = 0.0f, a = fabsf(x);
    if (a < 0.5f) r = -2.0f * a;
    else if (a < 1.5f) r = 0.5f * (2.0f * a - 3.0f);
    if (x < 0.0f) r *= -1.0f;
    return r;
}
/* taichi_utils.py:120-121 N_1 */
static inline float N1(float x) { return 1.0f - fabsf(x); }

/* taichi_utils.py:254-276 interp_2 (4-tap loop per axis, i outermost) */
static float interp2(sf_t f, float px, float py, float pz, float dx, float BLx, float BLy, float BLz) {
    float u = px / dx - BLx, v = py / dx - BLy, w = pz / dx - BLz;
    float s = fmaxr(1.0f, fminr(u, (float)(f.n0 - 2 - REF_EPS)));
    float t = fmaxr(1.0f, fminr(v, (float)(f.n1 - 2 - REF_EPS)));
    float l = fmaxr(1.0f, fminr(w, (float)(f.n2 - 2 - REF_EPS)));
    float iu = floorf(s), iv = floorf(t), iw = floorf(l);
    float acc = 0.0f;
    for (int i = -1; i < 3; i++)
        for (int j = -1; j < 3; j++)
            for (int k = -1; k < 3; k++) {
                float xx = s - (iu + (float)i), yy = t - (iv + (float)j), zz = l - (iw + (float)k);
                float val = samp(f, (int)(iu + (float)i), (int)(iv + (float)j), (int)(iw + (float)k));
                acc += val * N2(xx) * N2(yy) * N2(zz);
            }
    return acc;
}

/* taichi_utils.py:279-319 interp_grad_2 */
static float interp_grad2(sf_t f, float px, float py, float pz, float dx, float BLx, float BLy, float BLz,
                          float g[3]) {
    float u = px / dx - BLx, v = py / dx - BLy, w = pz / dx - BLz;
    float s = fmaxr(1.0f, fminr(u, (float)(f.n0 - 2 - REF_EPS)));
    float t = fmaxr(1.0f, fminr(v, (float)(f.n1 - 2 - REF_EPS)));
    float l = fmaxr(1.0f, fminr(w, (float)(f.n2 - 2 - REF_EPS)));
    float iu = floorf(s), iv = floorf(t), iw = floorf(l);
    float gx = 0.0f, gy = 0.0f, gz = 0.0f, acc = 0.0f;
    float inv = 1.0f / dx;
    for (int i = -1; i < 3; i++)
        for (int j = -1; j < 3; j++)
            for (int k = -1; k < 3; k++) {
                float xx = s - (iu + (float)i), yy = t - (iv + (float)j), zz = l - (iw + (float)k);
                float val = samp(f, (int)(iu + (float)i), (int)(iv + (float)j), (int)(iw + (float)k));
                gx += inv * (val * dN2(xx) * N2(yy) * N2(zz));
                gy += inv * (val * N2(xx) * dN2(yy) * N2(zz));
                gz += inv * (val * N2(xx) * N2(yy) * dN2(zz));
                acc += val * N2(xx) * N2(yy) * N2(zz);
            }
    g[0] = gx; g[1] = gy; g[2] = gz;
    return acc;
}

typedef struct { sf_t x, y, z; float dx; } mac_t;

static inline mac_t mac_make(const float *ux, const float *uy, const float *uz, int nx, int ny, int nz, float dx) {
    mac_t m;
    m.x.p = ux; m.x.n0 = nx + 1; m.x.n1 = ny; m.x.n2 = nz;
    m.y.p = uy; m.y.n0 = nx; m.y.n1 = ny + 1; m.y.n2 = nz;
    m.z.p = uz; m.z.n0 = nx; m.z.n1 = ny; m.z.n2 = nz + 1;
    m.dx = dx;
    return m;
}

/* taichi_utils.py:322-326 interp_u_MAC */
static inline void macv(const mac_t *m, const float p[3], float out[3]) {
    out[0] = interp2(m->x, p[0], p[1], p[2], m->dx, 0.0f, 0.5f, 0.5f);
    out[1] = interp2(m->y, p[0], p[1], p[2], m->dx, 0.5f, 0.0f, 0.5f);
    out[2] = interp2(m->z, p[0], p[1], p[2], m->dx, 0.5f, 0.5f, 0.0f);
}
/* taichi_utils.py:336-341 interp_u_MAC_grad: G rows = grad of u_x, u_y, u_z */
static inline void macg(const mac_t *m, const float p[3], float out[3], float G[3][3]) {
    out[0] = interp_grad2(m->x, p[0], p[1], p[2], m->dx, 0.0f, 0.5f, 0.5f, G[0]);
    out[1] = interp_grad2(m->y, p[0], p[1], p[2], m->dx, 0.5f, 0.0f, 0.5f, G[1]);
    out[2] = interp_grad2(m->z, p[0], p[1], p[2], m->dx, 0.5f, 0.5f, 0.0f, G[2]);
}

/* taichi_utils.py:172-198 interp_1 on a 4-channel cell field (BL 0.5) */
static void interp1_4(const float *f, int n0, int n1, int n2, const float p[3], float dx, float out[4]) {
    float u = p[0] / dx - 0.5f, v = p[1] / dx - 0.5f, w = p[2] / dx - 0.5f;
    float s = fmaxr(1.0f, fminr(u, (float)(n0 - 1 - REF_EPS)));
    float t = fmaxr(1.0f, fminr(v, (float)(n1 - 1 - REF_EPS)));
    float l = fmaxr(1.0f, fminr(w, (float)(n2 - 1 - REF_EPS)));
    float iu = floorf(s), iv = floorf(t), iw = floorf(l);
    float acc[4] = {0, 0, 0, 0};
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++)
            for (int k = 0; k < 2; k++) {
                float xx = s - (iu + (float)i), yy = t - (iv + (float)j), zz = l - (iw + (float)k);
                const float *val = samp_v(f, n0, n1, n2, 4, (int)(iu + i), (int)(iv + j), (int)(iw + k));
                float a = N1(xx), b = N1(yy), c = N1(zz);
                for (int q = 0; q < 4; q++) acc[q] += val[q] * a * b * c;
            }
    for (int q = 0; q < 4; q++) out[q] = acc[q];
}

/* taichi_utils.py:201-227 sample_min_max_1 on a 4-channel cell field */
static void minmax1_4(const float *f, int n0, int n1, int n2, const float p[3], float dx, float mn[4], float mx[4]) {
    float u = p[0] / dx - 0.5f, v = p[1] / dx - 0.5f, w = p[2] / dx - 0.5f;
    float s = fmaxr(1.0f, fminr(u, (float)(n0 - 1 - REF_EPS)));
    float t = fmaxr(1.0f, fminr(v, (float)(n1 - 1 - REF_EPS)));
    float l = fmaxr(1.0f, fminr(w, (float)(n2 - 1 - REF_EPS)));
    int iu = (int)floorf(s), iv = (int)floorf(t), iw = (int)floorf(l);
    const float *v0 = samp_v(f, n0, n1, n2, 4, iu, iv, iw);
    for (int q = 0; q < 4; q++) { mn[q] = v0[q]; mx[q] = v0[q]; }
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++)
            for (int k = 0; k < 2; k++) {
                const float *val = samp_v(f, n0, n1, n2, 4, iu + i, iv + j, iw + k);
                for (int q = 0; q < 4; q++) {
                    mn[q] = fminr(mn[q], val[q]);
                    mx[q] = fmaxr(mx[q], val[q]);
                }
            }
}

/* ------------------------------------------------------------------------ */
/* Hermite interpolation                                                     */
/* ------------------------------------------------------------------------ */
/* hermite.py:4-41 hermite_f / hermite_df / hermite_g / hermite_dg */
static inline float hf(float x) {
    float a = fabsf(x), r = 0.0f;
    if (a < 1.0f) r = 2.0f * (a * a * a) - 3.0f * (a * a) + 1.0f;
    return r;
}
static inline float hdf(float x) {
    float a = fabsf(x), r = 0.0f;
    if (a < 1.0f) r = 6.0f * (a * a) - 6.0f * a;
    if (x < 0.0f) r = -r;
    return r;
}
static inline float hg(float x) {
    float a = fabsf(x), r = 0.0f;
    if (a < 1.0f) r = (a * a * a) - 2.0f * (a * a) + a;
    if (x < 0.0f) r = -r;
    return r;
}
static inline float hdg(float x) {
    float a = fabsf(x), r = 0.0f;
    if (a < 1.0f) r = 3.0f * (a * a) - 4.0f * a + 1.0f;
    return r;
}

enum { HV_FD = 0, HV_GARM = 1, HV_FULL = 2 };

typedef struct {
    const float *psi;               /* vec3 cell field */
    const float *T[3];              /* rows: T_c = grad psi_c (vec3 cell fields) */
    const float *dT[3];             /* (psi_c,yz, psi_c,xz, psi_c,xy) (vec3) */
    const float *d2T[3];            /* psi_c,xyz (scalar) — ED8 only */
    int nx, ny, nz;
    float dx;
} map_t;

#define V3(f, i, j, k) samp_v((f), m->nx, m->ny, m->nz, 3, (i), (j), (k))

/* Hermite interpolation of psi_c at p; the three variants are
 *   HV_FD   interp_(grad_)hermite_fd_unroll       hermite.py:65-295
 *   HV_GARM interp_(grad_)hermite_garm_fd_unroll  hermite.py:299-456
 *   HV_FULL interp_(grad_)hermite                 hermite.py:460-607
 * Term order per accumulator follows the reference (value, grad*dx,
 * mixed second derivatives, triple derivative). */
static float hermite(int variant, const map_t *m, int c, const float p[3], float *grad) {
    float dx = m->dx;
    float u = p[0] / dx - 0.5f, v = p[1] / dx - 0.5f, w = p[2] / dx - 0.5f;
    float s = fmaxr(1.0f, fminr(u, (float)(m->nx - 2 - REF_EPS)));
    float t = fmaxr(1.0f, fminr(v, (float)(m->ny - 2 - REF_EPS)));
    float l = fmaxr(1.0f, fminr(w, (float)(m->nz - 2 - REF_EPS)));
    float iu = floorf(s), iv = floorf(t), iw = floorf(l);
    float acc = 0.0f, gx = 0.0f, gy = 0.0f, gz = 0.0f;
    const float *G = m->T[c], *GG = m->dT[c];
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++)
            for (int k = 0; k < 2; k++) {
                float xx = s - (iu + (float)i), yy = t - (iv + (float)j), zz = l - (iw + (float)k);
                float hxf = hf(xx), hxg = hg(xx), dhxf = hdf(xx), dhxg = hdg(xx);
                float hyf = hf(yy), hyg = hg(yy), dhyf = hdf(yy), dhyg = hdg(yy);
                float hzf = hf(zz), hzg = hg(zz), dhzf = hdf(zz), dhzg = hdg(zz);
                int ii = (int)(iu + (float)i), jj = (int)(iv + (float)j), kk = (int)(iw + (float)k);
                float terms[8];
                terms[0] = V3(m->psi, ii, jj, kk)[c];
                const float *g0 = V3(G, ii, jj, kk);
                terms[1] = g0[0] * dx; terms[2] = g0[1] * dx; terms[3] = g0[2] * dx;
                if (variant == HV_FD) {
                    /* hermite.py:104-148: FD cross terms of grad */
                    terms[4] = ((V3(G, ii, jj, kk + 1)[1] - V3(G, ii, jj, kk - 1)[1]) +
                                (V3(G, ii, jj + 1, kk)[2] - V3(G, ii, jj - 1, kk)[2])) / 4.0f * dx;
                    terms[5] = ((V3(G, ii, jj, kk + 1)[0] - V3(G, ii, jj, kk - 1)[0]) +
                                (V3(G, ii + 1, jj, kk)[2] - V3(G, ii - 1, jj, kk)[2])) / 4.0f * dx;
                    terms[6] = ((V3(G, ii, jj + 1, kk)[0] - V3(G, ii, jj - 1, kk)[0]) +
                                (V3(G, ii + 1, jj, kk)[1] - V3(G, ii - 1, jj, kk)[1])) / 4.0f * dx;
                    float v30 = ((V3(G, ii + 1, jj, kk + 1)[1] - V3(G, ii + 1, jj, kk - 1)[1]) +
                                 (V3(G, ii + 1, jj + 1, kk)[2] - V3(G, ii + 1, jj - 1, kk)[2])) / 4.0f;
                    float v31 = ((V3(G, ii - 1, jj, kk + 1)[1] - V3(G, ii - 1, jj, kk - 1)[1]) +
                                 (V3(G, ii - 1, jj + 1, kk)[2] - V3(G, ii - 1, jj - 1, kk)[2])) / 4.0f;
                    float v32 = ((V3(G, ii, jj + 1, kk + 1)[0] - V3(G, ii, jj + 1, kk - 1)[0]) +
                                 (V3(G, ii + 1, jj + 1, kk)[2] - V3(G, ii - 1, jj + 1, kk)[2])) / 4.0f;
                    float v33 = ((V3(G, ii, jj - 1, kk + 1)[0] - V3(G, ii, jj - 1, kk - 1)[0]) +
                                 (V3(G, ii + 1, jj - 1, kk)[2] - V3(G, ii - 1, jj - 1, kk)[2])) / 4.0f;
                    float v34 = ((V3(G, ii, jj + 1, kk + 1)[0] - V3(G, ii, jj - 1, kk + 1)[0]) +
                                 (V3(G, ii + 1, jj, kk + 1)[1] - V3(G, ii - 1, jj, kk + 1)[1])) / 4.0f;
                    float v35 = ((V3(G, ii, jj + 1, kk - 1)[0] - V3(G, ii, jj - 1, kk - 1)[0]) +
                                 (V3(G, ii + 1, jj, kk - 1)[1] - V3(G, ii - 1, jj, kk - 1)[1])) / 4.0f;
                    terms[7] = (v30 - v31 + v32 - v33 + v34 - v35) / 6.0f * dx;
                } else {
                    const float *gg = V3(GG, ii, jj, kk);
                    terms[4] = gg[0] * dx * dx; terms[5] = gg[1] * dx * dx; terms[6] = gg[2] * dx * dx;
                    if (variant == HV_GARM) {
                        /* hermite.py:346-351: FD of the stored mixed derivatives */
                        terms[7] = ((V3(GG, ii + 1, jj, kk)[0] - V3(GG, ii - 1, jj, kk)[0]) +
                                    (V3(GG, ii, jj + 1, kk)[1] - V3(GG, ii, jj - 1, kk)[1]) +
                                    (V3(GG, ii, jj, kk + 1)[2] - V3(GG, ii, jj, kk - 1)[2])) / 6.0f * dx * dx;
                    } else {
                        sf_t d3 = {m->d2T[c], m->nx, m->ny, m->nz};
                        terms[7] = samp(d3, ii, jj, kk) * dx * dx * dx;
                    }
                }
                /* basis per term: (x,y,z) factor choice f/g */
                const float bx[8] = {hxf, hxg, hxf, hxf, hxf, hxg, hxg, hxg};
                const float by[8] = {hyf, hyf, hyg, hyf, hyg, hyf, hyg, hyg};
                const float bz[8] = {hzf, hzf, hzf, hzg, hzg, hzg, hzf, hzg};
                const float dbx[8] = {dhxf, dhxg, dhxf, dhxf, dhxf, dhxg, dhxg, dhxg};
                const float dby[8] = {dhyf, dhyf, dhyg, dhyf, dhyg, dhyf, dhyg, dhyg};
                const float dbz[8] = {dhzf, dhzf, dhzf, dhzg, dhzg, dhzg, dhzf, dhzg};
                for (int q = 0; q < 8; q++) {
                    acc += terms[q] * bx[q] * by[q] * bz[q];
                    if (grad) {
                        gx += terms[q] * dbx[q] * by[q] * bz[q];
                        gy += terms[q] * bx[q] * dby[q] * bz[q];
                        gz += terms[q] * bx[q] * by[q] * dbz[q];
                    }
                }
            }
    if (grad) {
        float inv = 1.0f / dx;
        grad[0] = gx * inv; grad[1] = gy * inv; grad[2] = gz * inv;
    }
    return acc;
}

/* ------------------------------------------------------------------------ */
/* RK4 marches                                                               */
/* ------------------------------------------------------------------------ */
/* hermite.py:786-803 advance_map_0 (RK4 of a point, velocity only) */
static void rk4_pos(const mac_t *mac, float psi[3], float dt) {
    float u1[3], u2[3], u3[3], u4[3], q[3];
    float h = 0.5f * dt;
    macv(mac, psi, u1);
    for (int c = 0; c < 3; c++) q[c] = psi[c] + h * u1[c];
    macv(mac, q, u2);
    for (int c = 0; c < 3; c++) q[c] = psi[c] + h * u2[c];
    macv(mac, q, u3);
    for (int c = 0; c < 3; c++) q[c] = psi[c] + dt * u3[c];
    macv(mac, q, u4);
    float w6 = dt * 1.0f / 6.0f;
    for (int c = 0; c < 3; c++) psi[c] = psi[c] + w6 * (u1[c] + 2.0f * u2[c] + 2.0f * u3[c] + u4[c]);
}

static inline void matvec(const float G[3][3], const float v[3], float o[3]) {
    for (int r = 0; r < 3; r++) o[r] = G[r][0] * v[0] + G[r][1] * v[1] + G[r][2] * v[2];
}

/* RK4 of a point with Jacobian columns C[a] (dC/dt = grad u . C), the
 * common body of hermite.py:806-860 advance_map_1_transpose_func (where
 * C are the transposed rows) and run_edge.py:337-357 advance_map (one
 * column per face). ncol columns are marched. */
static void rk4_jac(const mac_t *mac, float psi[3], float C[][3], int ncol, float dt) {
    float u[4][3], G[3][3], q[3], Cs[3][3], d[4][3][3];
    float h = 0.5f * dt;
    macg(mac, psi, u[0], G);
    for (int a = 0; a < ncol; a++) matvec(G, C[a], d[0][a]);
    for (int c = 0; c < 3; c++) q[c] = psi[c] + h * u[0][c];
    for (int a = 0; a < ncol; a++) for (int c = 0; c < 3; c++) Cs[a][c] = C[a][c] + h * d[0][a][c];
    macg(mac, q, u[1], G);
    for (int a = 0; a < ncol; a++) matvec(G, Cs[a], d[1][a]);
    for (int c = 0; c < 3; c++) q[c] = psi[c] + h * u[1][c];
    for (int a = 0; a < ncol; a++) for (int c = 0; c < 3; c++) Cs[a][c] = C[a][c] + h * d[1][a][c];
    macg(mac, q, u[2], G);
    for (int a = 0; a < ncol; a++) matvec(G, Cs[a], d[2][a]);
    for (int c = 0; c < 3; c++) q[c] = psi[c] + dt * u[2][c];
    for (int a = 0; a < ncol; a++) for (int c = 0; c < 3; c++) Cs[a][c] = C[a][c] + dt * d[2][a][c];
    macg(mac, q, u[3], G);
    for (int a = 0; a < ncol; a++) matvec(G, Cs[a], d[3][a]);
    float w6 = dt * 1.0f / 6.0f;
    for (int c = 0; c < 3; c++)
        psi[c] = psi[c] + w6 * (u[0][c] + 2.0f * u[1][c] + 2.0f * u[2][c] + u[3][c]);
    for (int a = 0; a < ncol; a++)
        for (int c = 0; c < 3; c++)
            C[a][c] = C[a][c] + w6 * (d[0][a][c] + 2.0f * d[1][a][c] + 2.0f * d[2][a][c] + d[3][a][c]);
}

/* hermite.py:806-860 on a point given as rows T (row c = grad psi_c). */
static void rk4_rows(const mac_t *mac, float psi[3], float T[3][3], float dt) {
    float C[3][3];
    for (int a = 0; a < 3; a++) for (int c = 0; c < 3; c++) C[a][c] = T[c][a];
    rk4_jac(mac, psi, C, 3, dt);
    for (int a = 0; a < 3; a++) for (int c = 0; c < 3; c++) T[c][a] = C[a][c];
}

/* hermite.py:959-980 interp_psi_hermite_garm_fd_unroll_func (and the
 * HV_FULL twin hermite.py:1006-1020): compose point p (with step Jacobian
 * rows Tn) through the accumulated map. */
static void compose(int variant, const map_t *m, float p[3], float Tn[3][3]) {
    float np3[3], To[3][3];
    for (int c = 0; c < 3; c++) np3[c] = hermite(variant, m, c, p, To[c]);
    float Tr[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) Tr[i][j] = To[i][0] * Tn[0][j] + To[i][1] * Tn[1][j] + To[i][2] * Tn[2][j];
    memcpy(Tn, Tr, sizeof(Tr));
    memcpy(p, np3, sizeof(np3));
}

static inline void cell_pos(int i, int j, int k, float dx, float X[3]) {
    X[0] = ((float)i + 0.5f) * dx; X[1] = ((float)j + 0.5f) * dx; X[2] = ((float)k + 0.5f) * dx;
}
static inline void face_pos(int axis, int i, int j, int k, float dx, float X[3]) {
    X[0] = ((float)i + (axis == 0 ? 0.0f : 0.5f)) * dx;
    X[1] = ((float)j + (axis == 1 ? 0.0f : 0.5f)) * dx;
    X[2] = ((float)k + (axis == 2 ? 0.0f : 0.5f)) * dx;
}

static const float ED4_OFF[4][3] = {{-1, -1, -1}, {1, 1, -1}, {-1, 1, 1}, {1, -1, 1}};   /* hermite.py:1446-1449 */
static const float ED8_OFF[8][3] = {                                                   /* hermite.py:716-723 */
    {-1, -1, -1}, {1, -1, -1}, {-1, 1, -1}, {1, 1, -1}, {-1, -1, 1}, {1, -1, 1}, {-1, 1, 1}, {1, 1, 1}};

/* hermite.py:1426-1521 advect_psi_garm_ed4_fusion_unroll: EDGE march.
 * Inputs: accumulated map (psi, T rows, dT); outputs to separate buffers. */
EXPORT void orc_march_edge(int nx, int ny, int nz, float dx, float dt, float epsilon,
                           const float *ux, const float *uy, const float *uz,
                           const float *psi, const float *Tx, const float *Ty, const float *Tz,
                           const float *dTx, const float *dTy, const float *dTz,
                           float *opsi, float *oTx, float *oTy, float *oTz,
                           float *odTx, float *odTy, float *odTz) {
    mac_t mac = mac_make(ux, uy, uz, nx, ny, nz, dx);
    map_t m = {psi, {Tx, Ty, Tz}, {dTx, dTy, dTz}, {0, 0, 0}, nx, ny, nz, dx};
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                float X[3];
                cell_pos(i, j, k, dx, X);
                float P[5][3], T[5][3][3];
                for (int q = 0; q < 5; q++) {
                    for (int c = 0; c < 3; c++) {
                        P[q][c] = q == 0 ? X[c] : X[c] + ED4_OFF[q - 1][c] * epsilon;
                        for (int d = 0; d < 3; d++) T[q][c][d] = (c == d) ? 1.0f : 0.0f;
                    }
                }
                for (int q = 0; q < 5; q++) rk4_rows(&mac, P[q], T[q], -dt);
                for (int q = 0; q < 5; q++) compose(HV_GARM, &m, P[q], T[q]);
                size_t o = ix3(i, j, k, ny, nz) * 3;
                float *Tp[3] = {oTx + o, oTy + o, oTz + o};
                float *dp[3] = {odTx + o, odTy + o, odTz + o};
                for (int c = 0; c < 3; c++) {
                    opsi[o + c] = P[0][c];
                    for (int d = 0; d < 3; d++) Tp[c][d] = T[0][c][d];
                }
                /* hermite.py:1049-1075 calc_ed4_garm_func, row c = T_c of the 4 points */
                float e8 = 8.0f;
                for (int c = 0; c < 3; c++) {
                    const float *t0 = T[1][c], *t1 = T[2][c], *t2 = T[3][c], *t3 = T[4][c];
                    dp[c][0] = ((-t0[1] - t1[1] + t2[1] + t3[1]) + (-t0[2] + t1[2] + t2[2] - t3[2])) / e8 / epsilon;
                    dp[c][1] = ((-t0[0] - t1[0] + t2[0] + t3[0]) + (-t0[2] + t1[2] - t2[2] + t3[2])) / e8 / epsilon;
                    dp[c][2] = ((-t0[0] + t1[0] + t2[0] - t3[0]) + (-t0[1] + t1[1] - t2[1] + t3[1])) / e8 / epsilon;
                }
            }
}

/* hermite.py:1375-1395 advect_ps_hermite_ed4_fd_unroll: ED4 march. */
EXPORT void orc_march_ed4(int nx, int ny, int nz, float dx, float dt, float epsilon,
                          const float *ux, const float *uy, const float *uz,
                          const float *psi, const float *Tx, const float *Ty, const float *Tz,
                          float *opsi, float *oTx, float *oTy, float *oTz) {
    mac_t mac = mac_make(ux, uy, uz, nx, ny, nz, dx);
    map_t m = {psi, {Tx, Ty, Tz}, {0, 0, 0}, {0, 0, 0}, nx, ny, nz, dx};
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                float X[3], P[4][3];
                cell_pos(i, j, k, dx, X);
                for (int q = 0; q < 4; q++) {
                    for (int c = 0; c < 3; c++) P[q][c] = X[c] + ED4_OFF[q][c] * epsilon;
                    rk4_pos(&mac, P[q], -dt);
                    float r[3];
                    for (int c = 0; c < 3; c++) r[c] = hermite(HV_FD, &m, c, P[q], NULL);
                    memcpy(P[q], r, sizeof(r));
                }
                /* hermite.py:1154-1177 calc_ed4_1 */
                size_t o = ix3(i, j, k, ny, nz) * 3;
                float px[3], py[3], pz[3];
                for (int c = 0; c < 3; c++) {
                    opsi[o + c] = (P[0][c] + P[1][c] + P[2][c] + P[3][c]) / 4.0f;
                    px[c] = (-P[0][c] + P[1][c] - P[2][c] + P[3][c]) / 4.0f / epsilon;
                    py[c] = (-P[0][c] + P[1][c] + P[2][c] - P[3][c]) / 4.0f / epsilon;
                    pz[c] = (-P[0][c] - P[1][c] + P[2][c] + P[3][c]) / 4.0f / epsilon;
                }
                float *Tp[3] = {oTx + o, oTy + o, oTz + o};
                for (int c = 0; c < 3; c++) { Tp[c][0] = px[c]; Tp[c][1] = py[c]; Tp[c][2] = pz[c]; }
            }
}

/* hermite.py:1290-1338 advect_ps_hermite_ed8: ED8 march. */
EXPORT void orc_march_ed8(int nx, int ny, int nz, float dx, float dt, float epsilon,
                          const float *ux, const float *uy, const float *uz,
                          const float *psi, const float *Tx, const float *Ty, const float *Tz,
                          const float *dTx, const float *dTy, const float *dTz,
                          const float *d2Tx, const float *d2Ty, const float *d2Tz,
                          float *opsi, float *oTx, float *oTy, float *oTz,
                          float *odTx, float *odTy, float *odTz, float *od2Tx, float *od2Ty, float *od2Tz) {
    mac_t mac = mac_make(ux, uy, uz, nx, ny, nz, dx);
    map_t m = {psi, {Tx, Ty, Tz}, {dTx, dTy, dTz}, {d2Tx, d2Ty, d2Tz}, nx, ny, nz, dx};
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                float X[3], P[8][3];
                cell_pos(i, j, k, dx, X);
                for (int q = 0; q < 8; q++) {
                    for (int c = 0; c < 3; c++) P[q][c] = X[c] + ED8_OFF[q][c] * epsilon;
                    rk4_pos(&mac, P[q], -dt);
                    float r[3];
                    for (int c = 0; c < 3; c++) r[c] = hermite(HV_FULL, &m, c, P[q], NULL);
                    memcpy(P[q], r, sizeof(r));
                }
                /* hermite.py:1098-1151 calc_ed8_3; P order 000,001,010,011,100,101,110,111 */
                size_t o = ix3(i, j, k, ny, nz);
                float ps[3], px[3], py[3], pz[3], pyz[3], pzx[3], pxy[3], pxyz[3];
                for (int c = 0; c < 3; c++) {
                    float a0 = P[0][c], a1 = P[1][c], a2 = P[2][c], a3 = P[3][c];
                    float a4 = P[4][c], a5 = P[5][c], a6 = P[6][c], a7 = P[7][c];
                    ps[c] = (a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7) / 8.0f;
                    px[c] = (-a0 + a1 - a2 + a3 - a4 + a5 - a6 + a7) / 8.0f / epsilon;
                    py[c] = (-a0 - a1 + a2 + a3 - a4 - a5 + a6 + a7) / 8.0f / epsilon;
                    pz[c] = (-a0 - a1 - a2 - a3 + a4 + a5 + a6 + a7) / 8.0f / epsilon;
                    pyz[c] = (a0 + a1 - a2 - a3 - a4 - a5 + a6 + a7) / 8.0f / epsilon / epsilon;
                    pzx[c] = (a0 - a1 + a2 - a3 - a4 + a5 - a6 + a7) / 8.0f / epsilon / epsilon;
                    pxy[c] = (a0 - a1 - a2 + a3 + a4 - a5 - a6 + a7) / 8.0f / epsilon / epsilon;
                    pxyz[c] = (-a0 + a1 + a2 - a3 + a4 - a5 - a6 + a7) / 8.0f / epsilon / epsilon / epsilon;
                }
                float *Tp[3] = {oTx + 3 * o, oTy + 3 * o, oTz + 3 * o};
                float *dp[3] = {odTx + 3 * o, odTy + 3 * o, odTz + 3 * o};
                float *d2p[3] = {od2Tx + o, od2Ty + o, od2Tz + o};
                for (int c = 0; c < 3; c++) {
                    opsi[3 * o + c] = ps[c];
                    Tp[c][0] = px[c]; Tp[c][1] = py[c]; Tp[c][2] = pz[c];
                    dp[c][0] = pyz[c]; dp[c][1] = pzx[c]; dp[c][2] = pxy[c];
                    *d2p[c] = pxyz[c];
                }
            }
}

/* hermite.py:1180-1256 calc_fd_3_from_grad: the mixed second derivatives of
 * each psi_c from central differences of its stored gradient row T_c (index
 * clamped at the walls, taichi_utils.py sample), then the triple derivative
 * from central differences of those.  The dT loops finish before the d2T
 * loops start (separate offloaded loops of one Taichi kernel). */
EXPORT void orc_calc_fd_3_from_grad(int nx, int ny, int nz, float dx,
                                    const float *Tx, const float *Ty, const float *Tz,
                                    float *dTx, float *dTy, float *dTz, float *d2Tx, float *d2Ty, float *d2Tz) {
    const float *T[3] = {Tx, Ty, Tz};
    float *dT[3] = {dTx, dTy, dTz};
    float *d2T[3] = {d2Tx, d2Ty, d2Tz};
    for (int c = 0; c < 3; c++) {
        const float *t = T[c];
#pragma omp parallel for collapse(2) schedule(static)
        for (int i = 0; i < nx; i++)
            for (int j = 0; j < ny; j++)
                for (int k = 0; k < nz; k++) {
#define TS(a, b, d) samp_v(t, nx, ny, nz, 3, (a), (b), (d))
                    float *o = dT[c] + 3 * ix3(i, j, k, ny, nz);
                    o[0] = ((TS(i, j, k + 1)[1] - TS(i, j, k - 1)[1]) + (TS(i, j + 1, k)[2] - TS(i, j - 1, k)[2])) / 4.0f / dx;
                    o[1] = ((TS(i, j, k + 1)[0] - TS(i, j, k - 1)[0]) + (TS(i + 1, j, k)[2] - TS(i - 1, j, k)[2])) / 4.0f / dx;
                    o[2] = ((TS(i, j + 1, k)[0] - TS(i, j - 1, k)[0]) + (TS(i + 1, j, k)[1] - TS(i - 1, j, k)[1])) / 4.0f / dx;
#undef TS
                }
    }
    for (int c = 0; c < 3; c++) {
        const float *t = dT[c];
#pragma omp parallel for collapse(2) schedule(static)
        for (int i = 0; i < nx; i++)
            for (int j = 0; j < ny; j++)
                for (int k = 0; k < nz; k++) {
#define DS(a, b, d) samp_v(t, nx, ny, nz, 3, (a), (b), (d))
                    d2T[c][ix3(i, j, k, ny, nz)] = ((DS(i + 1, j, k)[0] - DS(i - 1, j, k)[0]) +
                                                    (DS(i, j + 1, k)[1] - DS(i, j - 1, k)[1]) +
                                                    (DS(i, j, k + 1)[2] - DS(i, j, k - 1)[2])) / 6.0f / dx;
#undef DS
                }
    }
}

/* hermite.py:1398-1424 advect_ps_garm (the GE march, run_ge.py:220-230):
 * every cell centre is marched back by RK4 with its Jacobian from the
 * identity (reset_to_identity_1, advance_map_1_transpose with -dt,
 * hermite.py:643-654, 864-918), composed with the accumulated map by the full
 * stored-derivative Hermite (interp_psi_hermite_garm, hermite.py:1024-1046),
 * and dT, d2T of the new map come from calc_fd_3_from_grad. */
EXPORT void orc_march_ge(int nx, int ny, int nz, float dx, float dt,
                         const float *ux, const float *uy, const float *uz,
                         const float *psi, const float *Tx, const float *Ty, const float *Tz,
                         const float *dTx, const float *dTy, const float *dTz,
                         const float *d2Tx, const float *d2Ty, const float *d2Tz,
                         float *opsi, float *oTx, float *oTy, float *oTz,
                         float *odTx, float *odTy, float *odTz, float *od2Tx, float *od2Ty, float *od2Tz) {
    mac_t mac = mac_make(ux, uy, uz, nx, ny, nz, dx);
    map_t m = {psi, {Tx, Ty, Tz}, {dTx, dTy, dTz}, {d2Tx, d2Ty, d2Tz}, nx, ny, nz, dx};
    float *oT[3] = {oTx, oTy, oTz};
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                float P[3], T[3][3];
                cell_pos(i, j, k, dx, P);
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++) T[a][b] = a == b ? 1.0f : 0.0f;
                rk4_rows(&mac, P, T, -dt);
                compose(HV_FULL, &m, P, T);
                size_t o = ix3(i, j, k, ny, nz);
                for (int c = 0; c < 3; c++) {
                    opsi[3 * o + c] = P[c];
                    for (int d = 0; d < 3; d++) oT[c][3 * o + d] = T[c][d];
                }
            }
    orc_calc_fd_3_from_grad(nx, ny, nz, dx, oTx, oTy, oTz, odTx, odTy, odTz, od2Tx, od2Ty, od2Tz);
}

/* run_ed8.py:191-224 split_psi_hermite: full Hermite psi and Jacobian column
 * on each face grid (psi_f: vec3, T_f: vec3 = column `axis` of grad psi). */
EXPORT void orc_split_psi_hermite(int nx, int ny, int nz, float dx,
                                  const float *psi, const float *Tx, const float *Ty, const float *Tz,
                                  const float *dTx, const float *dTy, const float *dTz,
                                  const float *d2Tx, const float *d2Ty, const float *d2Tz,
                                  float *psi_fx, float *psi_fy, float *psi_fz,
                                  float *T_fx, float *T_fy, float *T_fz) {
    map_t m = {psi, {Tx, Ty, Tz}, {dTx, dTy, dTz}, {d2Tx, d2Ty, d2Tz}, nx, ny, nz, dx};
    float *PF[3] = {psi_fx, psi_fy, psi_fz}, *TF[3] = {T_fx, T_fy, T_fz};
    for (int a = 0; a < 3; a++) {
        int n0 = nx + (a == 0), n1 = ny + (a == 1), n2 = nz + (a == 2);
#pragma omp parallel for collapse(2) schedule(static)
        for (int i = 0; i < n0; i++)
            for (int j = 0; j < n1; j++)
                for (int k = 0; k < n2; k++) {
                    float X[3], G[3][3];
                    face_pos(a, i, j, k, dx, X);
                    size_t o = ix3(i, j, k, n1, n2) * 3;
                    for (int c = 0; c < 3; c++) PF[a][o + c] = hermite(HV_FULL, &m, c, X, G[c]);
                    for (int c = 0; c < 3; c++) TF[a][o + c] = G[c][a];
                }
    }
}

/* hermite.py:1578-1621 advect_u_semi_lagrangian (dt is the caller's, the
 * driver passes 0.5*curr_dt, run_edge.py:650-651). */
EXPORT void orc_advect_u_semi_lagrangian(int nx, int ny, int nz, float dx, float dt,
                                         const float *ux0, const float *uy0, const float *uz0,
                                         float *ux1, float *uy1, float *uz1) {
    mac_t mac = mac_make(ux0, uy0, uz0, nx, ny, nz, dx);
    float *OUT[3] = {ux1, uy1, uz1};
    for (int a = 0; a < 3; a++) {
        int n0 = nx + (a == 0), n1 = ny + (a == 1), n2 = nz + (a == 2);
#pragma omp parallel for collapse(2) schedule(static)
        for (int i = 0; i < n0; i++)
            for (int j = 0; j < n1; j++)
                for (int k = 0; k < n2; k++) {
                    float p1[3], v1[3], v2[3], v3[3], v4[3], v5[3], q[3];
                    face_pos(a, i, j, k, dx, p1);
                    macv(&mac, p1, v1);
                    for (int c = 0; c < 3; c++) q[c] = p1[c] - v1[c] * dt * 0.5f;
                    macv(&mac, q, v2);
                    for (int c = 0; c < 3; c++) q[c] = p1[c] - v2[c] * dt * 0.5f;
                    macv(&mac, q, v3);
                    for (int c = 0; c < 3; c++) q[c] = p1[c] - v3[c] * dt;
                    macv(&mac, q, v4);
                    for (int c = 0; c < 3; c++)
                        q[c] = p1[c] - (v1[c] + 2.0f * v2[c] + 2.0f * v3[c] + v4[c]) / 6.0f * dt;
                    macv(&mac, q, v5);
                    OUT[a][ix3(i, j, k, n1, n2)] = v5[a];
                }
    }
}

/* run_edge.py:337-357 advance_map: forward map phi and one Jacobian column F
 * on the face grid `axis` (in place). */
EXPORT void orc_advance_map(int nx, int ny, int nz, int axis, float dx, float dt,
                            const float *ux, const float *uy, const float *uz, float *phi, float *F) {
    mac_t mac = mac_make(ux, uy, uz, nx, ny, nz, dx);
    int n0 = nx + (axis == 0), n1 = ny + (axis == 1), n2 = nz + (axis == 2);
    size_t n = (size_t)n0 * n1 * n2;
#pragma omp parallel for schedule(static)
    for (size_t e = 0; e < n; e++) {
        float C[1][3];
        memcpy(C[0], F + 3 * e, sizeof(C[0]));
        rk4_jac(&mac, phi + 3 * e, C, 1, dt);
        memcpy(F + 3 * e, C[0], sizeof(C[0]));
    }
}

/* run_edge.py:361-373 map_u: u1_a = F_a . u0(phi_a) on each face grid */
EXPORT void orc_map_u(int nx, int ny, int nz, float dx,
                      const float *ux0, const float *uy0, const float *uz0,
                      float *ux1, float *uy1, float *uz1,
                      const float *Fx, const float *Fy, const float *Fz,
                      const float *phix, const float *phiy, const float *phiz) {
    mac_t mac = mac_make(ux0, uy0, uz0, nx, ny, nz, dx);
    float *OUT[3] = {ux1, uy1, uz1};
    const float *FF[3] = {Fx, Fy, Fz}, *PH[3] = {phix, phiy, phiz};
    for (int a = 0; a < 3; a++) {
        int n0 = nx + (a == 0), n1 = ny + (a == 1), n2 = nz + (a == 2);
        size_t n = (size_t)n0 * n1 * n2;
#pragma omp parallel for schedule(static)
        for (size_t e = 0; e < n; e++) {
            float v[3];
            macv(&mac, PH[a] + 3 * e, v);
            const float *f = FF[a] + 3 * e;
            OUT[a][e] = f[0] * v[0] + f[1] * v[1] + f[2] * v[2];
        }
    }
}

/* run_edge.py:377-417 map_u_psi (variant HV_GARM) and run_ed4.py:219-260
 * (variant HV_FD): u1_a(X_a) = (grad psi)^T column a . u0(psi(X_a)). */
EXPORT void orc_map_u_psi(int variant, int nx, int ny, int nz, float dx,
                          const float *ux0, const float *uy0, const float *uz0,
                          float *ux1, float *uy1, float *uz1,
                          const float *psi, const float *Tx, const float *Ty, const float *Tz,
                          const float *dTx, const float *dTy, const float *dTz) {
    mac_t mac = mac_make(ux0, uy0, uz0, nx, ny, nz, dx);
    map_t m = {psi, {Tx, Ty, Tz}, {dTx, dTy, dTz}, {0, 0, 0}, nx, ny, nz, dx};
    float *OUT[3] = {ux1, uy1, uz1};
    for (int a = 0; a < 3; a++) {
        int n0 = nx + (a == 0), n1 = ny + (a == 1), n2 = nz + (a == 2);
#pragma omp parallel for collapse(2) schedule(static)
        for (int i = 0; i < n0; i++)
            for (int j = 0; j < n1; j++)
                for (int k = 0; k < n2; k++) {
                    float X[3], G[3][3], P[3], v[3];
                    face_pos(a, i, j, k, dx, X);
                    for (int c = 0; c < 3; c++) P[c] = hermite(variant, &m, c, X, G[c]);
                    macv(&mac, P, v);
                    OUT[a][ix3(i, j, k, n1, n2)] = G[0][a] * v[0] + G[1][a] * v[1] + G[2][a] * v[2];
                }
    }
}

/* run_edge.py:430-440 split_to_mac then the 1/6 face average of
 * map_smoke_psi (run_edge.py:444-466) */
static void psi_center(int variant, const map_t *m, int i, int j, int k, float pc[3]) {
    float X[3], s[3] = {0, 0, 0};
    float acc[6][3];
    int q = 0;
    for (int a = 0; a < 3; a++)
        for (int side = 0; side < 2; side++) {
            face_pos(a, i + (a == 0 ? side : 0), j + (a == 1 ? side : 0), k + (a == 2 ? side : 0), m->dx, X);
            for (int c = 0; c < 3; c++) acc[q][c] = hermite(variant, m, c, X, NULL);
            q++;
        }
    for (int c = 0; c < 3; c++) {
        s[c] = acc[0][c] + acc[1][c] + acc[2][c] + acc[3][c] + acc[4][c] + acc[5][c];
        pc[c] = (1.0f / 6.0f) * s[c];
    }
}

/* run_edge.py:444-466 map_smoke_psi (HV_GARM) / run_ed4.py:293-310 (HV_FD) */
EXPORT void orc_map_smoke_psi(int variant, int nx, int ny, int nz, float dx, const float *smoke0, float *smoke1,
                              const float *psi, const float *Tx, const float *Ty, const float *Tz,
                              const float *dTx, const float *dTy, const float *dTz) {
    map_t m = {psi, {Tx, Ty, Tz}, {dTx, dTy, dTz}, {0, 0, 0}, nx, ny, nz, dx};
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                float pc[3];
                psi_center(variant, &m, i, j, k, pc);
                interp1_4(smoke0, nx, ny, nz, pc, dx, smoke1 + ix3(i, j, k, ny, nz) * 4);
            }
}

/* run_edge.py:481-505 clamp_smoke_psi (HV_GARM) / run_ed4.py:313-336 (HV_FD) */
EXPORT void orc_clamp_smoke_psi(int variant, int nx, int ny, int nz, float dx, const float *smoke0, float *smoke1,
                                const float *psi, const float *Tx, const float *Ty, const float *Tz,
                                const float *dTx, const float *dTy, const float *dTz) {
    map_t m = {psi, {Tx, Ty, Tz}, {dTx, dTy, dTz}, {0, 0, 0}, nx, ny, nz, dx};
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                float pc[3], mn[4], mx[4];
                psi_center(variant, &m, i, j, k, pc);
                minmax1_4(smoke0, nx, ny, nz, pc, dx, mn, mx);
                float *s = smoke1 + ix3(i, j, k, ny, nz) * 4;
                for (int q = 0; q < 4; q++) s[q] = fminr(fmaxr(s[q], mn[q]), mx[q]);
            }
}

static void phi_center(int nx, int ny, int nz, const float *px, const float *py, const float *pz,
                       int i, int j, int k, float pc[3]) {
    const float *a0 = px + ix3(i, j, k, ny, nz) * 3, *a1 = px + ix3(i + 1, j, k, ny, nz) * 3;
    const float *b0 = py + ix3(i, j, k, ny + 1, nz) * 3, *b1 = py + ix3(i, j + 1, k, ny + 1, nz) * 3;
    const float *c0 = pz + ix3(i, j, k, ny, nz + 1) * 3, *c1 = pz + ix3(i, j, k + 1, ny, nz + 1) * 3;
    for (int c = 0; c < 3; c++) pc[c] = (1.0f / 6.0f) * (a0[c] + a1[c] + b0[c] + b1[c] + c0[c] + c1[c]);
}

/* run_edge.py:421-427 map_smoke (forward face maps) */
EXPORT void orc_map_smoke(int nx, int ny, int nz, float dx, const float *smoke0, float *smoke1,
                          const float *phix, const float *phiy, const float *phiz) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                float pc[3];
                phi_center(nx, ny, nz, phix, phiy, phiz, i, j, k, pc);
                interp1_4(smoke0, nx, ny, nz, pc, dx, smoke1 + ix3(i, j, k, ny, nz) * 4);
            }
}

/* run_edge.py:470-477 clamp_smoke */
EXPORT void orc_clamp_smoke(int nx, int ny, int nz, float dx, const float *smoke0, float *smoke1,
                            const float *phix, const float *phiy, const float *phiz) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                float pc[3], mn[4], mx[4];
                phi_center(nx, ny, nz, phix, phiy, phiz, i, j, k, pc);
                minmax1_4(smoke0, nx, ny, nz, pc, dx, mn, mx);
                float *s = smoke1 + ix3(i, j, k, ny, nz) * 4;
                for (int q = 0; q < 4; q++) s[q] = fminr(fmaxr(s[q], mn[q]), mx[q]);
            }
}

/* run_edge.py:509-519 clamp_u on one face grid of shape (n0,n1,n2) */
EXPORT void orc_clamp_u(int n0, int n1, int n2, const float *u, const float *u1, float *u2) {
    sf_t f = {u1, n0, n1, n2};
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i < n0; i++)
        for (int j = 0; j < n1; j++)
            for (int k = 0; k < n2; k++) {
                float l = samp(f, i - 1, j, k), r = samp(f, i + 1, j, k);
                float b = samp(f, i, j - 1, k), t = samp(f, i, j + 1, k);
                float a = samp(f, i, j, k - 1), c = samp(f, i, j, k + 1);
                float mx = fmaxr(fmaxr(fmaxr(fmaxr(fmaxr(l, r), b), t), a), c);
                float mn = fminr(fminr(fminr(fminr(fminr(l, r), b), t), a), c);
                size_t e = ix3(i, j, k, n1, n2);
                u2[e] = fminr(fmaxr(u[e], mn), mx);
            }
}

/* run_edge.py:296-303 calc_max_speed */
EXPORT float orc_calc_max_speed(int nx, int ny, int nz, const float *ux, const float *uy, const float *uz) {
    float best = 1.e-3f;
#pragma omp parallel for collapse(2) reduction(max : best) schedule(static)
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                float u = 0.5f * (ux[ix3(i, j, k, ny, nz)] + ux[ix3(i + 1, j, k, ny, nz)]);
                float v = 0.5f * (uy[ix3(i, j, k, ny + 1, nz)] + uy[ix3(i, j + 1, k, ny + 1, nz)]);
                float w = 0.5f * (uz[ix3(i, j, k, ny, nz + 1)] + uz[ix3(i, j, k + 1, ny, nz + 1)]);
                float sp = sqrtf(u * u + v * v + w * w);
                if (sp > best) best = sp;
            }
    return best;
}

/* ------------------------------------------------------------------------ */
/* point samplers exported for the golden-vector tests                       */
/* ------------------------------------------------------------------------ */
EXPORT void orc_points_mac(int nx, int ny, int nz, float dx, const float *ux, const float *uy, const float *uz,
                           const float *pts, int n, float *v, float *vg, float *g) {
    mac_t mac = mac_make(ux, uy, uz, nx, ny, nz, dx);
    for (int e = 0; e < n; e++) {
        float G[3][3];
        macv(&mac, pts + 3 * e, v + 3 * e);
        macg(&mac, pts + 3 * e, vg + 3 * e, G);
        memcpy(g + 9 * e, G, sizeof(G));
    }
}

EXPORT void orc_points_dye(int nx, int ny, int nz, float dx, const float *smoke, const float *pts, int n,
                           float *lin, float *mn, float *mx) {
    for (int e = 0; e < n; e++) {
        interp1_4(smoke, nx, ny, nz, pts + 3 * e, dx, lin + 4 * e);
        minmax1_4(smoke, nx, ny, nz, pts + 3 * e, dx, mn + 4 * e, mx + 4 * e);
    }
}

EXPORT void orc_points_hermite(int variant, int nx, int ny, int nz, float dx, const float *psi,
                               const float *Tx, const float *Ty, const float *Tz,
                               const float *dTx, const float *dTy, const float *dTz,
                               const float *d2Tx, const float *d2Ty, const float *d2Tz,
                               const float *pts, int n, float *val, float *gval, float *grad) {
    map_t m = {psi, {Tx, Ty, Tz}, {dTx, dTy, dTz}, {d2Tx, d2Ty, d2Tz}, nx, ny, nz, dx};
    for (int e = 0; e < n; e++)
        for (int c = 0; c < 3; c++) {
            val[3 * e + c] = hermite(variant, &m, c, pts + 3 * e, NULL);
            gval[3 * e + c] = hermite(variant, &m, c, pts + 3 * e, grad + 9 * e + 3 * c);
        }
}

/* ------------------------------------------------------------------------ */
/* MGPCG (sim/mgpcg.py, sim/mgpcg_solid.py)                                  */
/* ------------------------------------------------------------------------ */
typedef struct {
    int L;
    int n[16][3];
    float *r[16], *z[16];
    int *bm[16]; /* solid mask per level (NULL for the plain solver) */
    float *x, *p, *Ap;
    int bt[3][2];
} mg_t;

static inline size_t lvl_size(const mg_t *s, int l) { return (size_t)s->n[l][0] * s->n[l][1] * s->n[l][2]; }

/* mgpcg.py:100-110 num_fluid_neighbors and mgpcg_solid.py:113-130 (with bm) */
static inline float nfluid(const mg_t *s, int l, int i, int j, int k) {
    const int *bm = s->bm[l];
    int n0 = s->n[l][0], n1 = s->n[l][1], n2 = s->n[l][2];
    int I[3] = {i, j, k}, D[3] = {n0, n1, n2};
    float num = 6.0f;
    for (int a = 0; a < 3; a++) {
        int lo[3] = {i, j, k}, hi[3] = {i, j, k};
        lo[a]--; hi[a]++;
        if (I[a] <= 0 && s->bt[a][0] == 2) num -= 1.0f;
        else if (bm && I[a] > 0 && bm[ix3(lo[0], lo[1], lo[2], n1, n2)] > 0) num -= 1.0f;
        if (I[a] >= D[a] - 1 && s->bt[a][1] == 2) num -= 1.0f;
        else if (bm && I[a] < D[a] - 1 && bm[ix3(hi[0], hi[1], hi[2], n1, n2)] > 0) num -= 1.0f;
    }
    return num;
}

/* mgpcg.py:88-98 neighbor_sum (right then left per axis) / mgpcg_solid.py:101-111 */
static inline float nsum(const mg_t *s, int l, const float *x, int i, int j, int k) {
    const int *bm = s->bm[l];
    int n1 = s->n[l][1], n2 = s->n[l][2];
    int I[3] = {i, j, k};
    float ret = 0.0f;
    for (int a = 0; a < 3; a++) {
        int hi[3] = {i, j, k}, lo[3] = {i, j, k};
        hi[a]++; lo[a]--;
        if (I[a] < s->n[l][a] - 1) {
            size_t e = ix3(hi[0], hi[1], hi[2], n1, n2);
            if (!bm || bm[e] <= 0) ret += x[e];
        }
        if (I[a] > 0) {
            size_t e = ix3(lo[0], lo[1], lo[2], n1, n2);
            if (!bm || bm[e] <= 0) ret += x[e];
        }
    }
    return ret;
}

static inline int fluid(const mg_t *s, int l, size_t e) { return !s->bm[l] || s->bm[l][e] <= 0; }

/* mgpcg.py:160-167 smooth (red/black phase) */
static void mg_smooth(mg_t *s, int l, int phase) {
    int n0 = s->n[l][0], n1 = s->n[l][1], n2 = s->n[l][2];
    float *z = s->z[l], *r = s->r[l];
#pragma omp parallel for collapse(2) schedule(static) if (n0 * n1 * n2 > OMP_MIN)
    for (int i = 0; i < n0; i++)
        for (int j = 0; j < n1; j++)
            for (int k = ((i + j + phase) & 1); k < n2; k += 2) {
                size_t e = ix3(i, j, k, n1, n2);
                if (!fluid(s, l, e)) continue;
                float mult = nfluid(s, l, i, j, k);
                z[e] = (r[e] + nsum(s, l, z, i, j, k)) / mult;
            }
}

/* mgpcg.py:147-153 restrict: r[l+1][I//2] += res * 1/(dim-1); the 8 children
 * of a coarse cell are summed in index order. */
static void mg_restrict(mg_t *s, int l) {
    int n1 = s->n[l][1], n2 = s->n[l][2];
    int c0 = s->n[l + 1][0], c1 = s->n[l + 1][1], c2 = s->n[l + 1][2];
    float *z = s->z[l], *r = s->r[l], *rc = s->r[l + 1];
#pragma omp parallel for collapse(2) schedule(static) if (c0 * c1 * c2 > OMP_MIN / 8)
    for (int I = 0; I < c0; I++)
        for (int J = 0; J < c1; J++)
            for (int K = 0; K < c2; K++) {
                float acc = 0.0f;
                for (int a = 0; a < 2; a++)
                    for (int b = 0; b < 2; b++)
                        for (int c = 0; c < 2; c++) {
                            int i = 2 * I + a, j = 2 * J + b, k = 2 * K + c;
                            size_t e = ix3(i, j, k, n1, n2);
                            if (!fluid(s, l, e)) continue;
                            float mult = nfluid(s, l, i, j, k);
                            float res = r[e] - (mult * z[e] - nsum(s, l, z, i, j, k));
                            acc += res * 1.0f / (3.0f - 1.0f);
                        }
                rc[ix3(I, J, K, c1, c2)] = acc;
            }
}

/* mgpcg.py:155-158 prolongate */
static void mg_prolong(mg_t *s, int l) {
    int n0 = s->n[l][0], n1 = s->n[l][1], n2 = s->n[l][2];
    int c1 = s->n[l + 1][1], c2 = s->n[l + 1][2];
#pragma omp parallel for collapse(2) schedule(static) if (n0 * n1 * n2 > OMP_MIN)
    for (int i = 0; i < n0; i++)
        for (int j = 0; j < n1; j++)
            for (int k = 0; k < n2; k++)
                s->z[l][ix3(i, j, k, n1, n2)] += s->z[l + 1][ix3(i / 2, j / 2, k / 2, c1, c2)];
}

/* mgpcg.py:177-195 apply_preconditioner (V-cycle) */
static void mg_vcycle(mg_t *s) {
    memset(s->z[0], 0, lvl_size(s, 0) * sizeof(float));
    for (int l = 0; l < s->L - 1; l++) {
        for (int it = 0; it < 2; it++) { mg_smooth(s, l, 0); mg_smooth(s, l, 1); }
        memset(s->z[l + 1], 0, lvl_size(s, l + 1) * sizeof(float));
        mg_restrict(s, l);
    }
    for (int it = 0; it < 20; it++) { mg_smooth(s, s->L - 1, 0); mg_smooth(s, s->L - 1, 1); }
    for (int l = s->L - 2; l >= 0; l--) {
        mg_prolong(s, l);
        for (int it = 0; it < 2; it++) { mg_smooth(s, l, 1); mg_smooth(s, l, 0); }
    }
}

/* mgpcg.py:126-130 reduce (the reference's float32 atomics; the oracle sums
 * in double, which any float32 reduction order approximates) */
static double mg_dot(const mg_t *s, const float *a, const float *b) {
    size_t n = lvl_size(s, 0);
    double acc = 0.0;
#pragma omp parallel for reduction(+ : acc) schedule(static)
    for (size_t e = 0; e < n; e++)
        if (fluid(s, 0, e)) acc += (double)a[e] * (double)b[e];
    return acc;
}

/* mgpcg.py:169-175 recenter: mean over all cells (solid cells included in the
 * solid solver, mgpcg_solid.py:197-202) */
static void mg_recenter(mg_t *s) {
    size_t n = lvl_size(s, 0);
    double acc = 0.0;
    float *r = s->r[0];
#pragma omp parallel for reduction(+ : acc) schedule(static)
    for (size_t e = 0; e < n; e++) acc += (double)r[e];
    float mean = (float)(acc / (double)n);
#pragma omp parallel for schedule(static)
    for (size_t e = 0; e < n; e++) r[e] -= mean;
}

static void mg_Ap(mg_t *s) {
    int n0 = s->n[0][0], n1 = s->n[0][1], n2 = s->n[0][2];
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i < n0; i++)
        for (int j = 0; j < n1; j++)
            for (int k = 0; k < n2; k++) {
                size_t e = ix3(i, j, k, n1, n2);
                if (!fluid(s, 0, e)) continue;
                s->Ap[e] = nfluid(s, 0, i, j, k) * s->p[e] - nsum(s, 0, s->p, i, j, k);
            }
}

/* mgpcg.py:197-283 solve (and mgpcg_solid.py:204-306): returns the iteration
 * index the reference prints at convergence, or -(iters) without it. */
static int mg_solve(mg_t *s, int max_iters, double abs_tol, double rel_tol, double *final_rTr) {
    size_t n = lvl_size(s, 0);
    const double eps = 1e-12;
    int all_neumann = (s->bt[0][0] + s->bt[0][1] + s->bt[1][0] + s->bt[1][1] + s->bt[2][0] + s->bt[2][1]) == 12;
    if (all_neumann) mg_recenter(s);
    mg_vcycle(s);
    /* update_p with beta = 0 (the field holds 0 from init) */
    for (size_t e = 0; e < n; e++)
        if (fluid(s, 0, e)) s->p[e] = s->z[0][e] + 0.0f * s->p[e];
    double old_zTr = (float)mg_dot(s, s->z[0], s->r[0]);
    double tol = abs_tol > old_zTr * rel_tol ? abs_tol : old_zTr * rel_tol;
    int it = 0;
    double rTr = 0.0;
    while (max_iters == -1 || it < max_iters) {
        mg_Ap(s);
        double pAp = (float)mg_dot(s, s->p, s->Ap);
        float alpha = (float)(old_zTr / (pAp + eps));
#pragma omp parallel for schedule(static)
        for (size_t e = 0; e < n; e++)
            if (fluid(s, 0, e)) {
                s->x[e] += alpha * s->p[e];
                s->r[0][e] -= alpha * s->Ap[e];
            }
        rTr = (float)mg_dot(s, s->r[0], s->r[0]);
        if (rTr < tol) {
            if (final_rTr) *final_rTr = rTr;
            return it;
        }
        if (all_neumann) mg_recenter(s);
        mg_vcycle(s);
        double new_zTr = (float)mg_dot(s, s->z[0], s->r[0]);
        float beta = (float)(new_zTr / (old_zTr + eps));
#pragma omp parallel for schedule(static)
        for (size_t e = 0; e < n; e++)
            if (fluid(s, 0, e)) s->p[e] = s->z[0][e] + beta * s->p[e];
        old_zTr = new_zTr;
        it++;
    }
    if (final_rTr) *final_rTr = rTr;
    return -it;
}

static int mg_init(mg_t *s, int nx, int ny, int nz, int base_level, const int *bt) {
    int mn = nx < ny ? nx : ny;
    mn = mn < nz ? mn : nz;
    int lg = 0;
    while ((1 << (lg + 1)) <= mn) lg++;
    s->L = lg - base_level + 1; /* mgpcg.py:34 */
    if (s->L < 1 || s->L > 16) return -1;
    for (int a = 0; a < 3; a++) for (int b = 0; b < 2; b++) s->bt[a][b] = bt[2 * a + b];
    for (int l = 0; l < s->L; l++) {
        s->n[l][0] = nx >> l; s->n[l][1] = ny >> l; s->n[l][2] = nz >> l;
        if (l > 0 && (s->n[l - 1][0] % 2 || s->n[l - 1][1] % 2 || s->n[l - 1][2] % 2)) return -2;
        s->r[l] = (float *)calloc(lvl_size(s, l), sizeof(float));
        s->z[l] = (float *)calloc(lvl_size(s, l), sizeof(float));
        s->bm[l] = NULL;
    }
    size_t n = lvl_size(s, 0);
    s->x = (float *)calloc(n, sizeof(float));
    s->p = (float *)calloc(n, sizeof(float));
    s->Ap = (float *)calloc(n, sizeof(float));
    return 0;
}

static void mg_free(mg_t *s) {
    for (int l = 0; l < s->L; l++) {
        free(s->r[l]); free(s->z[l]);
        if (l > 0) free(s->bm[l]);
    }
    free(s->x); free(s->p); free(s->Ap);
}

/* mgpcg.py:374-392 apply_bc (walls), + mgpcg_solid.py:344-356 (solid cells) */
static void apply_bc(int nx, int ny, int nz, const int *bt, float *ux, float *uy, float *uz,
                     const int *bm, const float *bvel) {
    for (int j = 0; j < ny; j++)
        for (int k = 0; k < nz; k++) {
            if (bt[0] == 2) ux[ix3(0, j, k, ny, nz)] = 0.0f;
            if (bt[1] == 2) ux[ix3(nx, j, k, ny, nz)] = 0.0f;
        }
    for (int i = 0; i < nx; i++)
        for (int k = 0; k < nz; k++) {
            if (bt[2] == 2) uy[ix3(i, 0, k, ny + 1, nz)] = 0.0f;
            if (bt[3] == 2) uy[ix3(i, ny, k, ny + 1, nz)] = 0.0f;
        }
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++) {
            if (bt[4] == 2) uz[ix3(i, j, 0, ny, nz + 1)] = 0.0f;
            if (bt[5] == 2) uz[ix3(i, j, nz, ny, nz + 1)] = 0.0f;
        }
    if (!bm) return;
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                size_t e = ix3(i, j, k, ny, nz);
                if (bm[e] <= 0) continue;
                const float *v = bvel + 3 * e;
                ux[ix3(i, j, k, ny, nz)] = v[0];
                ux[ix3(i + 1, j, k, ny, nz)] = v[0];
                uy[ix3(i, j, k, ny + 1, nz)] = v[1];
                uy[ix3(i, j + 1, k, ny + 1, nz)] = v[1];
                uz[ix3(i, j, k, ny, nz + 1)] = v[2];
                uz[ix3(i, j, k + 1, ny, nz + 1)] = v[2];
            }
}

/* mgpcg.py:394-404 divergence (no 1/dx) */
static void divergence(int nx, int ny, int nz, const float *ux, const float *uy, const float *uz, float *div,
                       const int *bm) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                size_t e = ix3(i, j, k, ny, nz);
                if (bm && bm[e] > 0) { div[e] = 0.0f; continue; }
                float vl = ux[ix3(i, j, k, ny, nz)], vr = ux[ix3(i + 1, j, k, ny, nz)];
                float vb = uy[ix3(i, j, k, ny + 1, nz)], vt = uy[ix3(i, j + 1, k, ny + 1, nz)];
                float va = uz[ix3(i, j, k, ny, nz + 1)], vc = uz[ix3(i, j, k + 1, ny, nz + 1)];
                div[e] = vr - vl + vt - vb + vc - va;
            }
}

/* mgpcg.py:406-432 subtract_grad_p (+ the force buffer of
 * subtract_grad_p_with_buffer, mgpcg.py:448-479, when f* != NULL) */
static void subtract_grad_p(int nx, int ny, int nz, const float *p, float *ux, float *uy, float *uz,
                            float *fx, float *fy, float *fz) {
    for (int a = 0; a < 3; a++) {
        int n0 = nx + (a == 0), n1 = ny + (a == 1), n2 = nz + (a == 2);
        float *u = a == 0 ? ux : (a == 1 ? uy : uz);
        float *f = a == 0 ? fx : (a == 1 ? fy : fz);
        int D = a == 0 ? nx : (a == 1 ? ny : nz);
#pragma omp parallel for collapse(2) schedule(static)
        for (int i = 0; i < n0; i++)
            for (int j = 0; j < n1; j++)
                for (int k = 0; k < n2; k++) {
                    int I[3] = {i, j, k};
                    int hi[3] = {clampi(i, 0, nx - 1), clampi(j, 0, ny - 1), clampi(k, 0, nz - 1)};
                    int lo[3] = {i, j, k};
                    lo[a] = clampi(I[a] - 1, 0, D - 1);
                    lo[(a + 1) % 3] = clampi(lo[(a + 1) % 3], 0, (a + 1) % 3 == 0 ? nx - 1 : ((a + 1) % 3 == 1 ? ny - 1 : nz - 1));
                    lo[(a + 2) % 3] = clampi(lo[(a + 2) % 3], 0, (a + 2) % 3 == 0 ? nx - 1 : ((a + 2) % 3 == 1 ? ny - 1 : nz - 1));
                    float pr = p[ix3(hi[0], hi[1], hi[2], ny, nz)];
                    float pl = p[ix3(lo[0], lo[1], lo[2], ny, nz)];
                    if (I[a] - 1 < 0) pl = 0.0f;
                    if (I[a] >= D) pr = 0.0f;
                    size_t e = ix3(i, j, k, n1, n2);
                    u[e] -= (pr - pl);
                    if (f) f[e] = -(pr - pl);
                }
    }
}

/* mgpcg.py:440-445 MGPCG_3.Poisson (fx may be NULL: Poisson_with_buffer when
 * set).  Returns the iteration count (see mg_solve); div/pressure optional
 * outputs (cell scalars). */
EXPORT int orc_poisson(int nx, int ny, int nz, int base_level, const int *bt, double abs_tol, double rel_tol,
                       int max_iters, float *ux, float *uy, float *uz, float *fx, float *fy, float *fz,
                       float *div_out, float *p_out, double *rTr_out) {
    mg_t s;
    memset(&s, 0, sizeof(s));
    if (mg_init(&s, nx, ny, nz, base_level, bt) != 0) return -100000;
    size_t n = lvl_size(&s, 0);
    float *div = (float *)malloc(n * sizeof(float));
    apply_bc(nx, ny, nz, bt, ux, uy, uz, NULL, NULL);
    divergence(nx, ny, nz, ux, uy, uz, div, NULL);
    for (size_t e = 0; e < n; e++) s.r[0][e] = div[e] * -1.0f; /* mgpcg.py:67-75 init(u_div, -1) */
    int it = mg_solve(&s, max_iters, abs_tol, rel_tol, rTr_out);
    subtract_grad_p(nx, ny, nz, s.x, ux, uy, uz, fx, fy, fz);
    apply_bc(nx, ny, nz, bt, ux, uy, uz, NULL, NULL);
    if (div_out) memcpy(div_out, div, n * sizeof(float));
    if (p_out) memcpy(p_out, s.x, n * sizeof(float));
    free(div);
    mg_free(&s);
    return it;
}

/* One V-cycle z = M^-1 r (mgpcg.py:177-195) and Ap (mgpcg.py:112-117) on the
 * fine level, for the preconditioner golden test. */
EXPORT int orc_vcycle(int nx, int ny, int nz, int base_level, const int *bt, const float *r, float *z, float *Ap) {
    mg_t s;
    memset(&s, 0, sizeof(s));
    if (mg_init(&s, nx, ny, nz, base_level, bt) != 0) return -1;
    size_t n = lvl_size(&s, 0);
    memcpy(s.r[0], r, n * sizeof(float));
    mg_vcycle(&s);
    memcpy(z, s.z[0], n * sizeof(float));
    memcpy(s.p, r, n * sizeof(float));
    mg_Ap(&s);
    memcpy(Ap, s.Ap, n * sizeof(float));
    int L = s.L;
    mg_free(&s);
    return L;
}

/* mgpcg_solid.py:87-97 downsample_bm */
static void downsample_bm(const mg_t *s, int l) {
    int c0 = s->n[l][0], c1 = s->n[l][1], c2 = s->n[l][2];
    int f1 = s->n[l - 1][1], f2 = s->n[l - 1][2];
    for (int I = 0; I < c0; I++)
        for (int J = 0; J < c1; J++)
            for (int K = 0; K < c2; K++) {
                int all = 1;
                for (int a = 0; a < 2; a++)
                    for (int b = 0; b < 2; b++)
                        for (int c = 0; c < 2; c++)
                            if (s->bm[l - 1][ix3(2 * I + a, 2 * J + b, 2 * K + c, f1, f2)] <= 0) all = 0;
                s->bm[l][ix3(I, J, K, c1, c2)] = all;
            }
}

/* mgpcg_solid.py:418-427 MGPCG_Solid_3.Poisson: walls, solid-cell velocities,
 * masked divergence with the >0-only mean correction (mgpcg_solid.py:359-383,
 * 422-424), masked MGPCG with tol=1e-12 absolute and max_iters=100. */
EXPORT int orc_poisson_solid(int nx, int ny, int nz, int base_level, const int *bt, const int *mask,
                             const float *bvel, double tol, int max_iters, float *ux, float *uy, float *uz,
                             float *div_out, float *p_out, int *bm1_out, int *bm2_out, double *div_sum_out) {
    mg_t s;
    memset(&s, 0, sizeof(s));
    if (mg_init(&s, nx, ny, nz, base_level, bt) != 0) return -100000;
    size_t n = lvl_size(&s, 0);
    s.bm[0] = (int *)mask;
    for (int l = 1; l < s.L; l++) s.bm[l] = (int *)calloc(lvl_size(&s, l), sizeof(int));
    float *div = (float *)malloc(n * sizeof(float));
    apply_bc(nx, ny, nz, bt, ux, uy, uz, mask, bvel);
    divergence(nx, ny, nz, ux, uy, uz, div, mask);
    float dsum = 0.0f; /* float32 accumulation as the reference's scalar field */
    int nfl = 0;
    double dsum_d = 0.0;
    for (size_t e = 0; e < n; e++)
        if (mask[e] <= 0) { dsum_d += div[e]; nfl++; }
    dsum = (float)dsum_d;
    if (div_sum_out) *div_sum_out = dsum;
    if (dsum > 0.0f && nfl > 0) {
        float avg = dsum / (float)nfl;
        for (size_t e = 0; e < n; e++)
            if (mask[e] <= 0) div[e] -= avg;
    }
    for (size_t e = 0; e < n; e++) s.r[0][e] = div[e] * -1.0f;
    for (int l = 1; l < s.L; l++) downsample_bm(&s, l);
    int it = mg_solve(&s, max_iters, tol, 0.0, NULL);
    subtract_grad_p(nx, ny, nz, s.x, ux, uy, uz, NULL, NULL, NULL);
    apply_bc(nx, ny, nz, bt, ux, uy, uz, mask, bvel);
    if (div_out) memcpy(div_out, div, n * sizeof(float));
    if (p_out) memcpy(p_out, s.x, n * sizeof(float));
    if (bm1_out && s.L > 1) memcpy(bm1_out, s.bm[1], lvl_size(&s, 1) * sizeof(int));
    if (bm2_out && s.L > 2) memcpy(bm2_out, s.bm[2], lvl_size(&s, 2) * sizeof(int));
    free(div);
    s.bm[0] = NULL;
    mg_free(&s);
    return it;
}

/* ------------------------------------------------------------------------ */
/* laden particles (sim/lp.py)                                               */
/* ------------------------------------------------------------------------ */
/* lp.py:6-29 update_particles_acc (G2P with interp_grad_2) */
EXPORT void orc_lp_acc(int nx, int ny, int nz, float dx, const float *ux, const float *uy, const float *uz,
                       const float *vel, const float *pos, float *acc, int num, int nmax, float dt, float St,
                       float gravity) {
    mac_t mac = mac_make(ux, uy, uz, nx, ny, nz, dx);
    for (int e = 0; e < nmax; e++) {
        float *a = acc + 3 * e;
        a[0] = a[1] = a[2] = 0.0f;
        if (e >= num) continue;
        float kk = 1.0f / St, v[3], G[3][3];
        macg(&mac, pos + 3 * e, v, G);
        a[1] += gravity;
        for (int c = 0; c < 3; c++) a[c] -= kk * (vel[3 * e + c] - v[c]);
        for (int c = 0; c < 3; c++) a[c] /= (1.0f + kk * dt);
    }
}

/* lp.py:32-70 update_particles_velocity */
EXPORT void orc_lp_velocity(const float *acc, float *vel, const float *pos, float dt, float dx, int num,
                            float Lx, float Ly, float Lz) {
    for (int e = 0; e < num; e++) {
        float *v = vel + 3 * e;
        const float *p = pos + 3 * e;
        for (int c = 0; c < 3; c++) v[c] += acc[3 * e + c] * dt;
        if (p[1] < dx && v[1] < 0) v[1] = 0.0f;
        if (p[1] > Ly - 3 * dx && v[1] > 0) v[1] = 0.0f;
        if (p[0] < 3 * dx && v[0] < 0) v[0] = 0.0f;
        if (p[0] > Lx - 3 * dx && v[0] > 0) v[0] = 0.0f;
        if (p[2] < 3 * dx && v[2] < 0) v[2] = 0.0f;
        if (p[2] > Lz - 3 * dx && v[2] > 0) v[2] = 0.0f;
    }
}

/* lp.py:73-97 calculate_velocity_diff */
EXPORT void orc_lp_vel_diff(int nx, int ny, int nz, float dx, const float *ux, const float *uy, const float *uz,
                            const float *vel, float *vdiff, const float *pos, int num, float St, float dens,
                            float erad) {
    mac_t mac = mac_make(ux, uy, uz, nx, ny, nz, dx);
    float eratio = 1.0f / (erad * erad * erad);
    for (int e = 0; e < num; e++) {
        float kk = 1.0f / St * dens * eratio, v[3], G[3][3];
        macg(&mac, pos + 3 * e, v, G);
        for (int c = 0; c < 3; c++) vdiff[3 * e + c] = kk * (vel[3 * e + c] - v[c]);
    }
}

/* lp.py:100-156 laden_particles_back_with_computing_particle (P2G scatter of
 * the drag with quadratic B-spline weights onto the three face grids) */
EXPORT void orc_lp_p2g(int nx, int ny, int nz, float dx, float *dragx, float *dragy, float *dragz,
                       const float *vdiff, const float *pos, const float *rad, int num, float lrad,
                       float Lx, float Ly, float Lz) {
    memset(dragx, 0, (size_t)(nx + 1) * ny * nz * sizeof(float));
    memset(dragy, 0, (size_t)nx * (ny + 1) * nz * sizeof(float));
    memset(dragz, 0, (size_t)nx * ny * (nz + 1) * sizeof(float));
    float *D[3] = {dragx, dragy, dragz};
    for (int e = 0; e < num; e++) {
        const float *p = pos + 3 * e;
        if (p[0] < 3 * dx || p[1] < 3 * dx || p[2] < 3 * dx || p[0] > Lx - 3 * dx || p[1] > Ly - 3 * dx ||
            p[2] > Lz - 3 * dx)
            continue;
        float g[3] = {p[0] / dx, p[1] / dx, p[2] / dx};
        float r = rad[e];
        float scale = r * r * r / (lrad * lrad * lrad);
        for (int a = 0; a < 3; a++) {
            int base[3];
            float off[3];
            for (int c = 0; c < 3; c++) {
                off[c] = (c == a) ? 0.0f : 0.5f;
                base[c] = (int)(g[c] - off[c]);
            }
            int n0 = nx + (a == 0), n1 = ny + (a == 1), n2 = nz + (a == 2);
            for (int oi = -1; oi < 3; oi++)
                for (int oj = -1; oj < 3; oj++)
                    for (int ok = -1; ok < 3; ok++) {
                        int f0 = base[0] + oi, f1 = base[1] + oj, f2 = base[2] + ok;
                        if (f0 < 0 || f0 >= n0 || f1 < 0 || f1 >= n1 || f2 < 0 || f2 >= n2) continue;
                        float w = N2(g[0] - (float)f0 - off[0]) * N2(g[1] - (float)f1 - off[1]) *
                                  N2(g[2] - (float)f2 - off[2]);
                        D[a][ix3(f0, f1, f2, n1, n2)] += vdiff[3 * e + a] * w * scale;
                    }
        }
    }
}

/* lp.py:158-181 update_particles_position */
EXPORT void orc_lp_position(const float *vel, float *pos, float dt, int num, float Lx, float Ly, float Lz) {
    float L[3] = {Lx, Ly, Lz};
    for (int e = 0; e < num; e++)
        for (int c = 0; c < 3; c++) {
            float *p = pos + 3 * e + c;
            *p += vel[3 * e + c] * dt;
            if (*p < 0) *p = 0.0f;
            if (*p > L[c]) *p = L[c];
        }
}

/* lp.py:183-219 calculate_viscous_force on one face grid */
EXPORT void orc_lp_viscous(int n0, int n1, int n2, float dx, float Re, const float *u, float *vis) {
    sf_t f = {u, n0, n1, n2};
    float nu = 1.0f / Re;
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i < n0; i++)
        for (int j = 0; j < n1; j++)
            for (int k = 0; k < n2; k++)
                vis[ix3(i, j, k, n1, n2)] =
                    nu * (samp(f, i + 1, j, k) + samp(f, i - 1, j, k) + samp(f, i, j + 1, k) + samp(f, i, j - 1, k) +
                          samp(f, i, j, k + 1) + samp(f, i, j, k - 1) + -6.0f * samp(f, i, j, k)) / dx / dx;
}

/* ------------------------------------------------------------------------ */
/* initial conditions                                                        */
/* ------------------------------------------------------------------------ */
/* init_conditions.py:11-36 add_vortex_ring_and_smoke (accumulates into u
 * (vec3 cells) and the dye's 4th channel, then thresholds the dye). */
EXPORT void orc_add_vortex_ring(int nx, int ny, int nz, float dx, float w, float rad, float delta, const float *cc,
                                const float *ex, const float *ey, float *u, float *smoke, const float *color,
                                int num_samples) {
    const float PI = 3.14159265358979323846f;
    float curve = (2.0f * PI * rad) / (float)num_samples;
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                float X[3];
                cell_pos(i, j, k, dx, X);
                size_t e = ix3(i, j, k, ny, nz);
                for (int l = 0; l < num_samples; l++) {
                    float th = (float)l / (float)num_samples * 2.0f * PI;
                    float ct = cosf(th), st = sinf(th), ps[3], d[3], wv[3];
                    for (int c = 0; c < 3; c++) ps[c] = rad * (ct * ex[c] + st * ey[c]) + cc[c];
                    for (int c = 0; c < 3; c++) d[c] = X[c] - ps[c];
                    float r = sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                    for (int c = 0; c < 3; c++) wv[c] = w * (-st * ex[c] + ct * ey[c]);
                    float q = r / delta;
                    float fac = curve * (-1.0f / (4.0f * PI * (r * r * r)) * (1.0f - expf(-(q * q * q))));
                    float cr[3] = {d[1] * wv[2] - d[2] * wv[1], d[2] * wv[0] - d[0] * wv[2], d[0] * wv[1] - d[1] * wv[0]};
                    for (int c = 0; c < 3; c++) u[3 * e + c] += fac * cr[c];
                    smoke[4 * e + 3] += curve * expf(-(q * q * q));
                }
                float *s = smoke + 4 * e;
                if (s[3] > 0.002f) { s[3] = 1.0f; s[0] = color[0]; s[1] = color[1]; s[2] = color[2]; }
                else { s[0] = s[1] = s[2] = s[3] = 0.0f; }
            }
}

/* taichi_utils.py:103-116 split_central_vector */
EXPORT void orc_split_central_vector(int nx, int ny, int nz, const float *vc, float *ux, float *uy, float *uz) {
    for (int i = 0; i <= nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                const float *r = vc + 3 * ix3(clampi(i, 0, nx - 1), j, k, ny, nz);
                const float *l = vc + 3 * ix3(clampi(i - 1, 0, nx - 1), j, k, ny, nz);
                ux[ix3(i, j, k, ny, nz)] = 0.5f * (r[0] + l[0]);
            }
    for (int i = 0; i < nx; i++)
        for (int j = 0; j <= ny; j++)
            for (int k = 0; k < nz; k++) {
                const float *t = vc + 3 * ix3(i, clampi(j, 0, ny - 1), k, ny, nz);
                const float *b = vc + 3 * ix3(i, clampi(j - 1, 0, ny - 1), k, ny, nz);
                uy[ix3(i, j, k, ny + 1, nz)] = 0.5f * (t[1] + b[1]);
            }
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k <= nz; k++) {
                const float *c = vc + 3 * ix3(i, j, clampi(k, 0, nz - 1), ny, nz);
                const float *a = vc + 3 * ix3(i, j, clampi(k - 1, 0, nz - 1), ny, nz);
                uz[ix3(i, j, k, ny, nz + 1)] = 0.5f * (c[2] + a[2]);
            }
}
