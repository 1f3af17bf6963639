// Shared device code for the EDGE sm_100a library: field geometry, the
// quadratic B-spline MAC sampler, the trilinear dye sampler, the three cubic
// Hermite flow-map interpolants and the RK4 point marches.
//
// Layout (identical to the reference's ti.field / to_numpy() order): scalar
// fields are row-major (i, j, k) with k fastest; vec3/vec4 fields store their
// components last (AoS).  Face grids of an (nx, ny, nz) cell grid are u_x
// (nx+1, ny, nz), u_y (nx, ny+1, nz), u_z (nx, ny, nz+1).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/edge_b200.h"

#define EDGE_HD __host__ __device__ __forceinline__
#define EDGE_D __device__ __forceinline__

namespace edge {

// taichi_utils.py:3 eps = 1e-6.  The reference clamps sample coordinates to
// [1, dim-2-eps] (B-spline, Hermite) or [1, dim-1-eps] (trilinear); Taichi
// folds that Python constant in double and narrows it to float32, so at
// dim >= ~64 the bound is exactly dim-2 (resp. dim-1).  Host code computes the
// bounds the same way and passes them in.
static inline float clamp_bound(int dim, int minus) { return (float)((double)(dim - minus) - 1e-6); }

EDGE_HD int idx3(int i, int j, int k, int n1, int n2) { return (i * n1 + j) * n2 + k; }
// x / dx as the reference writes it; when dx is a power of two (every grid
// spacing 1/res or 256/res of the drivers) the quotient is the exact scaling
// x * (1/dx), so the multiply gives the same float
static inline bool pow2f(float x) {
    int e;
    return x > 0.0f && frexpf(x, &e) == 0.5f;
}
EDGE_D float over_dx(float x, float dx, float inv_dx, bool pow2) { return pow2 ? x * inv_dx : x / dx; }
// A sampler struct with its power-of-two flag fixed at compile time: the hot
// kernels are built for both cases (P2 = pow2f(dx), chosen at launch), so
// over_dx is the exact multiply by 1/dx or the division with no run-time
// select between them (which made every sample evaluate the division too).
template <bool P2, class T>
EDGE_D T with_pow2(T s) {
    s.pow2 = P2 ? 1 : 0;
    return s;
}
// v[a] with constant indices only (a run-time index into a register array
// or a kernel-parameter array puts it in local memory)
EDGE_D float sel3(const float v[3], int a) { return a == 0 ? v[0] : (a == 1 ? v[1] : v[2]); }
EDGE_D int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// ---------------------------------------------------------------------------
// quadratic B-spline (taichi_utils.py:230-251) evaluated separably on the three
// non-zero taps of each axis
// ---------------------------------------------------------------------------
EDGE_D float N2(float x) {
    float a = fabsf(x);
    float r = 0.0f;
    if (a < 0.5f) r = 0.75f - a * a;
    else if (a < 1.5f) { float t = 1.5f - a; r = 0.5f * (t * t); }
    return r;
}
EDGE_D float dN2(float x) {
    float a = fabsf(x);
    float r = 0.0f;
    if (a < 0.5f) r = -2.0f * a;
    else if (a < 1.5f) r = 0.5f * (2.0f * a - 3.0f);
    return x < 0.0f ? -r : r;
}

// One axis of interp_2 / interp_grad_2 (taichi_utils.py:254-319): the clamped
// grid coordinate, the first of the three taps that carry weight (the 4th tap
// of the reference's -1..2 loop is always zero) and their weights.
struct Axis3 {
    int base;
    float w[3];
    float dw[3];
};
template <bool GRAD>
EDGE_D Axis3 bspline_axis(float u, float hi) {
    Axis3 a;
    float s = fmaxf(1.0f, fminf(u, hi));
    float iu = floorf(s);
    const float bf = (s - iu < 0.5f) ? iu - 1.0f : iu;  // the first tap, an integer held exactly
    float x0 = s - bf;
    a.base = (int)bf;
    // x0 lies in [0.5, 1.5) (exactly: s - b is exact), so the branches of
    // N2 / dN2 at x0, x0 - 1 and x0 - 2 are known: the same operations as the
    // general functions, without their compares.  The third tap's zero
    // branch (|x0 - 2| = 1.5, i.e. x0 = 0.5) needs no select either: there
    // t2 = 0 and 2 a2 - 3 = 0, so the polynomial gives the same zero; and
    // |x1| |x1| = x1 x1, sign(x1) * (-2 |x1|) = -2 x1 exactly.
    const float x1 = x0 - 1.0f, x2 = x0 - 2.0f;  // x1 in [-0.5, 0.5), x2 in [-1.5, -0.5)
    const float t0 = 1.5f - x0, a2 = -x2, t2 = 1.5f - a2;
    a.w[0] = 0.5f * (t0 * t0);
    a.w[1] = 0.75f - x1 * x1;
    a.w[2] = 0.5f * (t2 * t2);
    if (GRAD) {
        a.dw[0] = 0.5f * (2.0f * x0 - 3.0f);
        a.dw[1] = -2.0f * x1;
        a.dw[2] = -(0.5f * (2.0f * a2 - 3.0f));
    }
    return a;
}

// 27-tap separable contraction of one scalar field; g receives the gradient
// (already multiplied by 1/dx) when GRAD.
template <bool GRAD>
EDGE_D float bspline_sum(const float* __restrict__ f, int n1, int n2, const Axis3& X, const Axis3& Y,
                         const Axis3& Z, float inv_dx, float* g) {
    float v = 0.0f, gx = 0.0f, gy = 0.0f, gz = 0.0f;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        float cv = 0.0f, cy = 0.0f, cz = 0.0f;
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const float* row = f + idx3(X.base + i, Y.base + j, Z.base, n1, n2);
            float q0 = __ldg(row), q1 = __ldg(row + 1), q2 = __ldg(row + 2);
            float a = Z.w[0] * q0 + Z.w[1] * q1 + Z.w[2] * q2;
            cv += Y.w[j] * a;
            if (GRAD) {
                float dz = Z.dw[0] * q0 + Z.dw[1] * q1 + Z.dw[2] * q2;
                cy += Y.dw[j] * a;
                cz += Y.w[j] * dz;
            }
        }
        v += X.w[i] * cv;
        if (GRAD) {
            gx += X.dw[i] * cv;
            gy += X.w[i] * cy;
            gz += X.w[i] * cz;
        }
    }
    if (GRAD) {
        g[0] = gx * inv_dx;
        g[1] = gy * inv_dx;
        g[2] = gz * inv_dx;
    }
    return v;
}

// MAC velocity field + the clamp bounds of its three staggered components.
struct Mac {
    const float* __restrict__ u[3];
    int nx, ny, nz;
    float dx, inv_dx;
    int pow2;      // dx is a power of two
    float hi0[3];  // axis d, BL = 0   (the face field normal to d): dim = n_d + 1
    float hi5[3];  // axis d, BL = 0.5 (a face field tangential to d): dim = n_d
};

static inline Mac make_mac(const float* ux, const float* uy, const float* uz, int nx, int ny, int nz, float dx) {
    Mac m;
    m.u[0] = ux; m.u[1] = uy; m.u[2] = uz;
    m.nx = nx; m.ny = ny; m.nz = nz;
    m.dx = dx; m.inv_dx = 1.0f / dx; m.pow2 = pow2f(dx);
    int n[3] = {nx, ny, nz};
    for (int d = 0; d < 3; d++) {
        m.hi0[d] = clamp_bound(n[d] + 1, 2);
        m.hi5[d] = clamp_bound(n[d], 2);
    }
    return m;
}

// interp_u_MAC / interp_u_MAC_grad (taichi_utils.py:322-341).  G rows are the
// gradients of u_x, u_y, u_z.
template <bool GRAD>
EDGE_D void mac_sample(const Mac& m, const float p[3], float v[3], float G[3][3]) {
    float q[3] = {over_dx(p[0], m.dx, m.inv_dx, m.pow2), over_dx(p[1], m.dx, m.inv_dx, m.pow2),
                  over_dx(p[2], m.dx, m.inv_dx, m.pow2)};
    Axis3 A0[3], A5[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        A0[d] = bspline_axis<GRAD>(q[d], m.hi0[d]);
        A5[d] = bspline_axis<GRAD>(q[d] - 0.5f, m.hi5[d]);
    }
    v[0] = bspline_sum<GRAD>(m.u[0], m.ny, m.nz, A0[0], A5[1], A5[2], m.inv_dx, GRAD ? G[0] : nullptr);
    v[1] = bspline_sum<GRAD>(m.u[1], m.ny + 1, m.nz, A5[0], A0[1], A5[2], m.inv_dx, GRAD ? G[1] : nullptr);
    v[2] = bspline_sum<GRAD>(m.u[2], m.ny, m.nz + 1, A5[0], A5[1], A0[2], m.inv_dx, GRAD ? G[2] : nullptr);
}

// Component a of interp_u_MAC alone (mac_sample's arithmetic for that
// component): the semi-Lagrangian advection keeps only the face's own
// component of its last sample.
EDGE_D float mac_sample_comp(const Mac& m, const float p[3], int a) {
    float q[3] = {over_dx(p[0], m.dx, m.inv_dx, m.pow2), over_dx(p[1], m.dx, m.inv_dx, m.pow2),
                  over_dx(p[2], m.dx, m.inv_dx, m.pow2)};
    Axis3 A[3];
#pragma unroll
    for (int d = 0; d < 3; d++)
        A[d] = d == a ? bspline_axis<false>(q[d], m.hi0[d]) : bspline_axis<false>(q[d] - 0.5f, m.hi5[d]);
    if (a == 0) return bspline_sum<false>(m.u[0], m.ny, m.nz, A[0], A[1], A[2], m.inv_dx, nullptr);
    if (a == 1) return bspline_sum<false>(m.u[1], m.ny + 1, m.nz, A[0], A[1], A[2], m.inv_dx, nullptr);
    return bspline_sum<false>(m.u[2], m.ny, m.nz + 1, A[0], A[1], A[2], m.inv_dx, nullptr);
}

// ---------------------------------------------------------------------------
// trilinear dye sampler on 4-channel cell fields (taichi_utils.py:172-227)
// ---------------------------------------------------------------------------
struct Dye {
    int nx, ny, nz;
    float dx, inv_dx;
    int pow2;
    float hi[3];  // dim-1-eps
};
static inline Dye make_dye(int nx, int ny, int nz, float dx) {
    Dye d;
    d.nx = nx; d.ny = ny; d.nz = nz; d.dx = dx; d.inv_dx = 1.0f / dx; d.pow2 = pow2f(dx);
    d.hi[0] = clamp_bound(nx, 1);
    d.hi[1] = clamp_bound(ny, 1);
    d.hi[2] = clamp_bound(nz, 1);
    return d;
}
struct Lin8 {
    int i0, j0, k0, i1, j1, k1;
    float wx[2], wy[2], wz[2];
};
EDGE_D Lin8 lin_setup(const Dye& d, const float p[3]) {
    Lin8 L;
    float s[3];
    float u[3] = {over_dx(p[0], d.dx, d.inv_dx, d.pow2) - 0.5f, over_dx(p[1], d.dx, d.inv_dx, d.pow2) - 0.5f,
                  over_dx(p[2], d.dx, d.inv_dx, d.pow2) - 0.5f};
#pragma unroll
    for (int a = 0; a < 3; a++) s[a] = fmaxf(1.0f, fminf(u[a], d.hi[a]));
    float iu = floorf(s[0]), iv = floorf(s[1]), iw = floorf(s[2]);
    L.i0 = (int)iu; L.j0 = (int)iv; L.k0 = (int)iw;
    // sample() clamps the +1 corner (it can reach dim when s hits the bound)
    L.i1 = min(L.i0 + 1, d.nx - 1);
    L.j1 = min(L.j0 + 1, d.ny - 1);
    L.k1 = min(L.k0 + 1, d.nz - 1);
    L.wx[0] = 1.0f - fabsf(s[0] - iu); L.wx[1] = 1.0f - fabsf(s[0] - (iu + 1.0f));
    L.wy[0] = 1.0f - fabsf(s[1] - iv); L.wy[1] = 1.0f - fabsf(s[1] - (iv + 1.0f));
    L.wz[0] = 1.0f - fabsf(s[2] - iw); L.wz[1] = 1.0f - fabsf(s[2] - (iw + 1.0f));
    return L;
}
EDGE_D float4 ld4(const float* __restrict__ f, int e) { return __ldg(reinterpret_cast<const float4*>(f) + e); }

EDGE_D float4 dye_interp(const float* __restrict__ f, const Dye& d, const Lin8& L) {
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int c = 0; c < 8; c++) {
        int a = c >> 2, b = (c >> 1) & 1, q = c & 1;
        float4 v = ld4(f, idx3(a ? L.i1 : L.i0, b ? L.j1 : L.j0, q ? L.k1 : L.k0, d.ny, d.nz));
        float w = L.wx[a] * L.wy[b] * L.wz[q];
        acc.x += v.x * w; acc.y += v.y * w; acc.z += v.z * w; acc.w += v.w * w;
    }
    return acc;
}
EDGE_D void dye_minmax(const float* __restrict__ f, const Dye& d, const Lin8& L, float4& mn, float4& mx) {
#pragma unroll
    for (int c = 0; c < 8; c++) {
        int a = c >> 2, b = (c >> 1) & 1, q = c & 1;
        float4 v = ld4(f, idx3(a ? L.i1 : L.i0, b ? L.j1 : L.j0, q ? L.k1 : L.k0, d.ny, d.nz));
        if (c == 0) { mn = v; mx = v; }
        else {
            mn.x = fminf(mn.x, v.x); mn.y = fminf(mn.y, v.y); mn.z = fminf(mn.z, v.z); mn.w = fminf(mn.w, v.w);
            mx.x = fmaxf(mx.x, v.x); mx.y = fmaxf(mx.y, v.y); mx.z = fmaxf(mx.z, v.z); mx.w = fmaxf(mx.w, v.w);
        }
    }
}
EDGE_D float4 clamp4(float4 v, float4 lo, float4 hi) {
    return make_float4(fminf(fmaxf(v.x, lo.x), hi.x), fminf(fmaxf(v.y, lo.y), hi.y), fminf(fmaxf(v.z, lo.z), hi.z),
                       fminf(fmaxf(v.w, lo.w), hi.w));
}

// ---------------------------------------------------------------------------
// cubic Hermite flow-map interpolation (hermite.py:4-607)
// ---------------------------------------------------------------------------
enum Variant { HV_FD = EDGE_HERMITE_FD, HV_GARM = EDGE_HERMITE_GARM, HV_FULL = EDGE_HERMITE_FULL };

// Flow-map fields on the cell grid: psi (vec3), rows T_c = grad psi_c (vec3),
// dT_c = (psi_c,yz, psi_c,xz, psi_c,xy) (vec3) and d2T_c = psi_c,xyz (scalar).
struct MapF {
    const float* __restrict__ psi;
    const float* __restrict__ T[3];
    const float* __restrict__ dT[3];
    const float* __restrict__ d2T[3];
    int nx, ny, nz;
    float dx, inv_dx;
    int pow2;
    float hi[3];  // dim-2-eps
};
static inline MapF make_map(const float* psi, const float* const T[3], const float* const dT[3],
                            const float* const d2T[3], int nx, int ny, int nz, float dx) {
    MapF m;
    m.psi = psi;
    for (int c = 0; c < 3; c++) {
        m.T[c] = T[c];
        m.dT[c] = dT ? dT[c] : nullptr;
        m.d2T[c] = d2T ? d2T[c] : nullptr;
    }
    m.nx = nx; m.ny = ny; m.nz = nz; m.dx = dx; m.inv_dx = 1.0f / dx; m.pow2 = pow2f(dx);
    m.hi[0] = clamp_bound(nx, 2);
    m.hi[1] = clamp_bound(ny, 2);
    m.hi[2] = clamp_bound(nz, 2);
    return m;
}

// Basis of one axis at the two corners (i = 0, 1): hermite_f/g and their
// derivatives at x = s - (iu + i).
struct HAxis {
    int c0, cm, cp, cpp;   // iu, iu-1, iu+1, iu+2 (clamped as sample() does)
    float f[2], g[2], df[2], dg[2];
};
// hermite_f/g and derivatives at x with |x| <= 1 (haxis passes x in [0, 1)
// and [-1, 0)).  The reference's |x| >= 1 branch gives 0; at |x| = 1 every
// polynomial below is exactly 0 as well, so no select is needed.
EDGE_D void hbasis(float x, float& f, float& g, float& df, float& dg) {
    float a = fabsf(x);
    float a2 = a * a, a3 = a2 * a;
    f = 2.0f * a3 - 3.0f * a2 + 1.0f;
    float gg = a3 - 2.0f * a2 + a;
    float dff = 6.0f * a2 - 6.0f * a;
    dg = 3.0f * a2 - 4.0f * a + 1.0f;
    g = x < 0.0f ? -gg : gg;
    df = x < 0.0f ? -dff : dff;
}
EDGE_D HAxis haxis(float u, float hi, int n) {
    HAxis h;
    float s = fmaxf(1.0f, fminf(u, hi));
    float iu = floorf(s);
    int b = (int)iu;
    h.c0 = b;
    h.cm = b - 1;
    h.cp = min(b + 1, n - 1);
    h.cpp = min(b + 2, n - 1);
    hbasis(s - iu, h.f[0], h.g[0], h.df[0], h.dg[0]);
    hbasis(s - (iu + 1.0f), h.f[1], h.g[1], h.df[1], h.dg[1]);
    return h;
}

EDGE_D float ldv(const float* __restrict__ f, int e, int c) { return __ldg(f + 3 * e + c); }

// The 8 Hermite coefficients t[a][b][c] (a, b, c = 0 for f, 1 for g basis on
// x, y, z) of component `comp` at corner (ii, jj, kk); term scaling as in the
// reference (value, grad*dx, mixed*dx^2, triple*dx^3).
template <int VARIANT>
EDGE_D void hcoef(const MapF& m, int comp, int ii, int jj, int kk, int im, int ip, int jm, int jp, int km, int kp,
                  float t[8]) {
    const int n1 = m.ny, n2 = m.nz;
    const float dx = m.dx;
    const float* __restrict__ G = m.T[comp];
    int e = idx3(ii, jj, kk, n1, n2);
    t[0] = ldv(m.psi, e, comp);                  // fff
    t[4] = ldv(G, e, 0) * dx;                    // gff
    t[2] = ldv(G, e, 1) * dx;                    // fgf
    t[1] = ldv(G, e, 2) * dx;                    // ffg
    if (VARIANT == HV_FD) {
        // hermite.py:104-148 (FD of the stored gradient)
        int ekp = idx3(ii, jj, kp, n1, n2), ekm = idx3(ii, jj, km, n1, n2);
        int ejp = idx3(ii, jp, kk, n1, n2), ejm = idx3(ii, jm, kk, n1, n2);
        int eip = idx3(ip, jj, kk, n1, n2), eim = idx3(im, jj, kk, n1, n2);
        t[3] = ((ldv(G, ekp, 1) - ldv(G, ekm, 1)) + (ldv(G, ejp, 2) - ldv(G, ejm, 2))) / 4.0f * dx;   // fgg
        t[5] = ((ldv(G, ekp, 0) - ldv(G, ekm, 0)) + (ldv(G, eip, 2) - ldv(G, eim, 2))) / 4.0f * dx;   // gfg
        t[6] = ((ldv(G, ejp, 0) - ldv(G, ejm, 0)) + (ldv(G, eip, 1) - ldv(G, eim, 1))) / 4.0f * dx;   // ggf
        float v30 = ((ldv(G, idx3(ip, jj, kp, n1, n2), 1) - ldv(G, idx3(ip, jj, km, n1, n2), 1)) +
                     (ldv(G, idx3(ip, jp, kk, n1, n2), 2) - ldv(G, idx3(ip, jm, kk, n1, n2), 2))) / 4.0f;
        float v31 = ((ldv(G, idx3(im, jj, kp, n1, n2), 1) - ldv(G, idx3(im, jj, km, n1, n2), 1)) +
                     (ldv(G, idx3(im, jp, kk, n1, n2), 2) - ldv(G, idx3(im, jm, kk, n1, n2), 2))) / 4.0f;
        float v32 = ((ldv(G, idx3(ii, jp, kp, n1, n2), 0) - ldv(G, idx3(ii, jp, km, n1, n2), 0)) +
                     (ldv(G, idx3(ip, jp, kk, n1, n2), 2) - ldv(G, idx3(im, jp, kk, n1, n2), 2))) / 4.0f;
        float v33 = ((ldv(G, idx3(ii, jm, kp, n1, n2), 0) - ldv(G, idx3(ii, jm, km, n1, n2), 0)) +
                     (ldv(G, idx3(ip, jm, kk, n1, n2), 2) - ldv(G, idx3(im, jm, kk, n1, n2), 2))) / 4.0f;
        float v34 = ((ldv(G, idx3(ii, jp, kp, n1, n2), 0) - ldv(G, idx3(ii, jm, kp, n1, n2), 0)) +
                     (ldv(G, idx3(ip, jj, kp, n1, n2), 1) - ldv(G, idx3(im, jj, kp, n1, n2), 1))) / 4.0f;
        float v35 = ((ldv(G, idx3(ii, jp, km, n1, n2), 0) - ldv(G, idx3(ii, jm, km, n1, n2), 0)) +
                     (ldv(G, idx3(ip, jj, km, n1, n2), 1) - ldv(G, idx3(im, jj, km, n1, n2), 1))) / 4.0f;
        t[7] = (v30 - v31 + v32 - v33 + v34 - v35) / 6.0f * dx;  // ggg
    } else {
        const float* __restrict__ GG = m.dT[comp];
        t[3] = ldv(GG, e, 0) * dx * dx;  // fgg
        t[5] = ldv(GG, e, 1) * dx * dx;  // gfg
        t[6] = ldv(GG, e, 2) * dx * dx;  // ggf
        if (VARIANT == HV_GARM) {
            // hermite.py:346-351 (FD of the stored mixed derivatives)
            t[7] = ((ldv(GG, idx3(ip, jj, kk, n1, n2), 0) - ldv(GG, idx3(im, jj, kk, n1, n2), 0)) +
                    (ldv(GG, idx3(ii, jp, kk, n1, n2), 1) - ldv(GG, idx3(ii, jm, kk, n1, n2), 1)) +
                    (ldv(GG, idx3(ii, jj, kp, n1, n2), 2) - ldv(GG, idx3(ii, jj, km, n1, n2), 2))) / 6.0f * dx * dx;
        } else {
            t[7] = __ldg(m.d2T[comp] + e) * dx * dx * dx;  // hermite.py:508-509
        }
    }
}

// Hermite value (and gradient, already divided by dx, when GRAD) of all three
// components of psi at p.  Tensor-product evaluation: the 64 coefficients of
// the 2x2x2 corner stencil are contracted axis by axis (z, then y, then x).
template <int VARIANT, bool GRAD>
EDGE_D void hermite3(const MapF& m, const float p[3], float val[3], float grad[3][3]) {
    float q[3] = {over_dx(p[0], m.dx, m.inv_dx, m.pow2) - 0.5f, over_dx(p[1], m.dx, m.inv_dx, m.pow2) - 0.5f,
                  over_dx(p[2], m.dx, m.inv_dx, m.pow2) - 0.5f};
    HAxis X = haxis(q[0], m.hi[0], m.nx), Y = haxis(q[1], m.hi[1], m.ny), Z = haxis(q[2], m.hi[2], m.nz);
#pragma unroll
    for (int comp = 0; comp < 3; comp++) {
        float v = 0.0f, gx = 0.0f, gy = 0.0f, gz = 0.0f;
#pragma unroll
        for (int i = 0; i < 2; i++) {
            int ii = i ? X.cp : X.c0, im = i ? X.c0 : X.cm, ip = i ? X.cpp : X.cp;
            // per x-corner partial sums over (j, b) and (k, c)
            float Ax[2] = {0.f, 0.f}, dAx[2] = {0.f, 0.f}, Bx[2] = {0.f, 0.f}, dBx[2] = {0.f, 0.f};
            // Ax[a] = sum_{j,b,k,c} Y Z t[a][b][c]; Bx: with dY; dAx: with dZ
#pragma unroll
            for (int j = 0; j < 2; j++) {
                int jj = j ? Y.cp : Y.c0, jm = j ? Y.c0 : Y.cm, jp = j ? Y.cpp : Y.cp;
#pragma unroll
                for (int k = 0; k < 2; k++) {
                    int kk = k ? Z.cp : Z.c0, km = k ? Z.c0 : Z.cm, kp = k ? Z.cpp : Z.cp;
                    float t[8];
                    hcoef<VARIANT>(m, comp, ii, jj, kk, im, ip, jm, jp, km, kp, t);
                    // contract z (c): P[a][b] = Zf t[a][b][0] + Zg t[a][b][1]
#pragma unroll
                    for (int a = 0; a < 2; a++) {
                        float P0 = Z.f[k] * t[a * 4 + 0] + Z.g[k] * t[a * 4 + 1];
                        float P1 = Z.f[k] * t[a * 4 + 2] + Z.g[k] * t[a * 4 + 3];
                        float Q = Y.f[j] * P0 + Y.g[j] * P1;
                        Ax[a] += Q;
                        if (GRAD) {
                            float dP0 = Z.df[k] * t[a * 4 + 0] + Z.dg[k] * t[a * 4 + 1];
                            float dP1 = Z.df[k] * t[a * 4 + 2] + Z.dg[k] * t[a * 4 + 3];
                            Bx[a] += Y.df[j] * P0 + Y.dg[j] * P1;
                            dAx[a] += Y.f[j] * dP0 + Y.g[j] * dP1;
                        }
                    }
                }
            }
            v += X.f[i] * Ax[0] + X.g[i] * Ax[1];
            if (GRAD) {
                gx += X.df[i] * Ax[0] + X.dg[i] * Ax[1];
                gy += X.f[i] * Bx[0] + X.g[i] * Bx[1];
                gz += X.f[i] * dAx[0] + X.g[i] * dAx[1];
            }
            (void)dBx;
        }
        val[comp] = v;
        if (GRAD) {
            float inv = 1.0f / m.dx;
            grad[comp][0] = gx * inv;
            grad[comp][1] = gy * inv;
            grad[comp][2] = gz * inv;
        }
    }
}

// ---------------------------------------------------------------------------
// packed map layout: float4 planes, one cell per float4, components (x, y, z)
// in .x .y .z:
//   plane 0: psi
//   planes 1..3: d psi / dx, d psi / dy, d psi / dz   (columns of grad psi)
//   planes 4..6: psi_yz, psi_xz, psi_xy               (EDGE dT, ED8 dT)
//   plane 7: psi_xyz                                   (ED8 d2T)
// One 128-bit load then serves all three components of a Hermite stencil
// point.  The ED4 and EDGE maps carry fewer state planes (4 and 7); their
// remaining planes hold the Hermite coefficients the reference derives by
// finite differences at every evaluation (ED4: the fgg, gfg, ggf, ggg terms
// from the gradient, hermite.py:104-148; EDGE: the ggg term from the mixed
// derivatives, hermite.py:346-351), computed once per map by k_coef_p up to
// their final multiplications by dx, which the evaluation applies.  The
// corners a Hermite evaluation visits are cells 1..n-1 of each axis and the
// reference's neighbour indices there are the cell's own +-1 clamped to the
// grid, so a per-cell table with clamped neighbours holds exactly the values
// the reference computes per corner.  Every packed map is 8 planes.
// ---------------------------------------------------------------------------
constexpr int kPlanesED4 = 4, kPlanesEDGE = 7, kPlanesED8 = 8;  // state planes
constexpr int kPlanesStored = 8;
// internal variants: ED4 / EDGE Hermite reading the precomputed planes
constexpr int HV_FD_P = 3, HV_GARM_P = 4;

struct MapP {
    const float4* __restrict__ g;  // planes, plane q at g + q * n
    int n;                          // cells
    int nx, ny, nz;
    float dx, inv_dx;
    int pow2;
    float hi[3];
};
static inline MapP make_mapp(const float* planes, int nx, int ny, int nz, float dx) {
    MapP m;
    m.g = reinterpret_cast<const float4*>(planes);
    m.n = nx * ny * nz;
    m.nx = nx; m.ny = ny; m.nz = nz; m.dx = dx; m.inv_dx = 1.0f / dx; m.pow2 = pow2f(dx);
    m.hi[0] = clamp_bound(nx, 2);
    m.hi[1] = clamp_bound(ny, 2);
    m.hi[2] = clamp_bound(nz, 2);
    return m;
}
EDGE_D float4 ldp(const MapP& m, int q, int e) { return __ldg(m.g + (size_t)q * m.n + e); }
EDGE_D float c4(const float4& v, int c) { return c == 0 ? v.x : (c == 1 ? v.y : v.z); }

// Coefficients t[comp][8] of the corner (ii, jj, kk) from the packed planes
// (same terms and scaling as hcoef).
template <int VARIANT>
EDGE_D void hcoef_p(const MapP& m, int ii, int jj, int kk, int im, int ip, int jm, int jp, int km, int kp,
                    float t[3][8]) {
    const int n1 = m.ny, n2 = m.nz;
    const float dx = m.dx;
    const int e = idx3(ii, jj, kk, n1, n2);
    float4 P = ldp(m, 0, e), G0 = ldp(m, 1, e), G1 = ldp(m, 2, e), G2 = ldp(m, 3, e);
#pragma unroll
    for (int c = 0; c < 3; c++) {
        t[c][0] = c4(P, c);
        t[c][4] = c4(G0, c) * dx;
        t[c][2] = c4(G1, c) * dx;
        t[c][1] = c4(G2, c) * dx;
    }
    if (VARIANT == HV_FD_P) {
        float4 A = ldp(m, 4, e), B = ldp(m, 5, e), C = ldp(m, 6, e), D = ldp(m, 7, e);
#pragma unroll
        for (int c = 0; c < 3; c++) {
            t[c][3] = c4(A, c) * dx;
            t[c][5] = c4(B, c) * dx;
            t[c][6] = c4(C, c) * dx;
            t[c][7] = c4(D, c) * dx;
        }
    } else if (VARIANT == HV_FD) {
        // hermite.py:104-148: FD of the stored gradient (plane 1+d = d psi/dx_d)
        const int ekp = idx3(ii, jj, kp, n1, n2), ekm = idx3(ii, jj, km, n1, n2);
        const int ejp = idx3(ii, jp, kk, n1, n2), ejm = idx3(ii, jm, kk, n1, n2);
        const int eip = idx3(ip, jj, kk, n1, n2), eim = idx3(im, jj, kk, n1, n2);
        float4 kp1 = ldp(m, 2, ekp), km1 = ldp(m, 2, ekm), kp0 = ldp(m, 1, ekp), km0 = ldp(m, 1, ekm);
        float4 jp2 = ldp(m, 3, ejp), jm2 = ldp(m, 3, ejm), jp0 = ldp(m, 1, ejp), jm0 = ldp(m, 1, ejm);
        float4 ip2 = ldp(m, 3, eip), im2 = ldp(m, 3, eim), ip1 = ldp(m, 2, eip), im1 = ldp(m, 2, eim);
        // triple term: v30..v35 (hermite.py:128-145)
        float4 a30 = ldp(m, 2, idx3(ip, jj, kp, n1, n2)), b30 = ldp(m, 2, idx3(ip, jj, km, n1, n2));
        float4 c30 = ldp(m, 3, idx3(ip, jp, kk, n1, n2)), d30 = ldp(m, 3, idx3(ip, jm, kk, n1, n2));
        float4 a31 = ldp(m, 2, idx3(im, jj, kp, n1, n2)), b31 = ldp(m, 2, idx3(im, jj, km, n1, n2));
        float4 c31 = ldp(m, 3, idx3(im, jp, kk, n1, n2)), d31 = ldp(m, 3, idx3(im, jm, kk, n1, n2));
        float4 a32 = ldp(m, 1, idx3(ii, jp, kp, n1, n2)), b32 = ldp(m, 1, idx3(ii, jp, km, n1, n2));
        float4 c32 = ldp(m, 3, idx3(ip, jp, kk, n1, n2)), d32 = ldp(m, 3, idx3(im, jp, kk, n1, n2));
        float4 a33 = ldp(m, 1, idx3(ii, jm, kp, n1, n2)), b33 = ldp(m, 1, idx3(ii, jm, km, n1, n2));
        float4 c33 = ldp(m, 3, idx3(ip, jm, kk, n1, n2)), d33 = ldp(m, 3, idx3(im, jm, kk, n1, n2));
        float4 a34 = ldp(m, 1, idx3(ii, jp, kp, n1, n2)), b34 = ldp(m, 1, idx3(ii, jm, kp, n1, n2));
        float4 c34 = ldp(m, 2, idx3(ip, jj, kp, n1, n2)), d34 = ldp(m, 2, idx3(im, jj, kp, n1, n2));
        float4 a35 = ldp(m, 1, idx3(ii, jp, km, n1, n2)), b35 = ldp(m, 1, idx3(ii, jm, km, n1, n2));
        float4 c35 = ldp(m, 2, idx3(ip, jj, km, n1, n2)), d35 = ldp(m, 2, idx3(im, jj, km, n1, n2));
#pragma unroll
        for (int c = 0; c < 3; c++) {
            t[c][3] = ((c4(kp1, c) - c4(km1, c)) + (c4(jp2, c) - c4(jm2, c))) / 4.0f * dx;
            t[c][5] = ((c4(kp0, c) - c4(km0, c)) + (c4(ip2, c) - c4(im2, c))) / 4.0f * dx;
            t[c][6] = ((c4(jp0, c) - c4(jm0, c)) + (c4(ip1, c) - c4(im1, c))) / 4.0f * dx;
            float v30 = ((c4(a30, c) - c4(b30, c)) + (c4(c30, c) - c4(d30, c))) / 4.0f;
            float v31 = ((c4(a31, c) - c4(b31, c)) + (c4(c31, c) - c4(d31, c))) / 4.0f;
            float v32 = ((c4(a32, c) - c4(b32, c)) + (c4(c32, c) - c4(d32, c))) / 4.0f;
            float v33 = ((c4(a33, c) - c4(b33, c)) + (c4(c33, c) - c4(d33, c))) / 4.0f;
            float v34 = ((c4(a34, c) - c4(b34, c)) + (c4(c34, c) - c4(d34, c))) / 4.0f;
            float v35 = ((c4(a35, c) - c4(b35, c)) + (c4(c35, c) - c4(d35, c))) / 4.0f;
            t[c][7] = (v30 - v31 + v32 - v33 + v34 - v35) / 6.0f * dx;
        }
    } else {
        float4 D0 = ldp(m, 4, e), D1 = ldp(m, 5, e), D2 = ldp(m, 6, e);
        if (VARIANT == HV_GARM_P) {
            float4 X3 = ldp(m, 7, e);
#pragma unroll
            for (int c = 0; c < 3; c++) t[c][7] = c4(X3, c) * dx * dx;
        } else if (VARIANT == HV_GARM) {
            float4 xp = ldp(m, 4, idx3(ip, jj, kk, n1, n2)), xm = ldp(m, 4, idx3(im, jj, kk, n1, n2));
            float4 yp = ldp(m, 5, idx3(ii, jp, kk, n1, n2)), ym = ldp(m, 5, idx3(ii, jm, kk, n1, n2));
            float4 zp = ldp(m, 6, idx3(ii, jj, kp, n1, n2)), zm = ldp(m, 6, idx3(ii, jj, km, n1, n2));
#pragma unroll
            for (int c = 0; c < 3; c++)
                t[c][7] = ((c4(xp, c) - c4(xm, c)) + (c4(yp, c) - c4(ym, c)) + (c4(zp, c) - c4(zm, c))) / 6.0f * dx *
                          dx;
        } else {
            float4 X3 = ldp(m, 7, e);
#pragma unroll
            for (int c = 0; c < 3; c++) t[c][7] = c4(X3, c) * dx * dx * dx;
        }
#pragma unroll
        for (int c = 0; c < 3; c++) {
            t[c][3] = c4(D0, c) * dx * dx;
            t[c][5] = c4(D1, c) * dx * dx;
            t[c][6] = c4(D2, c) * dx * dx;
        }
    }
}

// The coefficients of hcoef_p divided by dx^(number of g factors), for a
// power-of-two dx (every such scaling is then exact): the g basis functions
// carry the factor dx instead (hermite3p), which gives every product of the
// contraction the same value with 3 multiplications per corner instead of 33.
template <int VARIANT>
EDGE_D void hcoef_p_unscaled(const MapP& m, int ii, int jj, int kk, float t[3][8]) {
    const int e = idx3(ii, jj, kk, m.ny, m.nz);
    const float inv = m.inv_dx;
    float4 P = ldp(m, 0, e), G0 = ldp(m, 1, e), G1 = ldp(m, 2, e), G2 = ldp(m, 3, e);
    float4 A = ldp(m, 4, e), B = ldp(m, 5, e), C = ldp(m, 6, e), D = ldp(m, 7, e);
#pragma unroll
    for (int c = 0; c < 3; c++) {
        t[c][0] = c4(P, c);
        t[c][4] = c4(G0, c);
        t[c][2] = c4(G1, c);
        t[c][1] = c4(G2, c);
        if (VARIANT == HV_FD_P) {  // planes 4-7 hold the terms over dx (hcoef_p multiplies by dx once)
            t[c][3] = c4(A, c) * inv;
            t[c][5] = c4(B, c) * inv;
            t[c][6] = c4(C, c) * inv;
            t[c][7] = c4(D, c) * inv * inv;
        } else {
            t[c][3] = c4(A, c);
            t[c][5] = c4(B, c);
            t[c][6] = c4(C, c);
            t[c][7] = VARIANT == HV_GARM_P ? c4(D, c) * inv : c4(D, c);  // GARM_P plane 7 holds psi_xyz over dx
        }
    }
}

// hermite3 on the packed layout: the 8 corners are visited once and feed all
// three components.  GSEL >= 0 computes only column GSEL of the gradient
// (grad[c][GSEL]; the other columns are left unset) with the same arithmetic:
// the face map keeps only the derivative along the face's own axis.
template <int VARIANT, bool GRAD, int GSEL = -1>
EDGE_D void hermite3p(const MapP& m, const float p[3], float val[3], float grad[3][3]) {
    constexpr bool GX = GRAD && (GSEL < 0 || GSEL == 0);
    constexpr bool GY = GRAD && (GSEL < 0 || GSEL == 1);
    constexpr bool GZ = GRAD && (GSEL < 0 || GSEL == 2);
    float q[3] = {over_dx(p[0], m.dx, m.inv_dx, m.pow2) - 0.5f, over_dx(p[1], m.dx, m.inv_dx, m.pow2) - 0.5f,
                  over_dx(p[2], m.dx, m.inv_dx, m.pow2) - 0.5f};
    HAxis X = haxis(q[0], m.hi[0], m.nx), Y = haxis(q[1], m.hi[1], m.ny), Z = haxis(q[2], m.hi[2], m.nz);
    // power-of-two dx: the g basis functions carry dx and the coefficients
    // come unscaled (hcoef_p_unscaled); the same products, fewer multiplies
    const bool fold = (VARIANT == HV_FD_P || VARIANT == HV_GARM_P || VARIANT == HV_FULL) && m.pow2;
    if (fold) {
#pragma unroll
        for (int c = 0; c < 2; c++) {
            X.g[c] *= m.dx; X.dg[c] *= m.dx;
            Y.g[c] *= m.dx; Y.dg[c] *= m.dx;
            Z.g[c] *= m.dx; Z.dg[c] *= m.dx;
        }
    }
    float v[3] = {0.f, 0.f, 0.f}, gx[3] = {0.f, 0.f, 0.f}, gy[3] = {0.f, 0.f, 0.f}, gz[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int i = 0; i < 2; i++) {
        int ii = i ? X.cp : X.c0, im = i ? X.c0 : X.cm, ip = i ? X.cpp : X.cp;
        float Ax[3][2] = {{0.f, 0.f}, {0.f, 0.f}, {0.f, 0.f}};
        float Bx[3][2] = {{0.f, 0.f}, {0.f, 0.f}, {0.f, 0.f}};
        float dAx[3][2] = {{0.f, 0.f}, {0.f, 0.f}, {0.f, 0.f}};
#pragma unroll
        for (int j = 0; j < 2; j++) {
            int jj = j ? Y.cp : Y.c0, jm = j ? Y.c0 : Y.cm, jp = j ? Y.cpp : Y.cp;
#pragma unroll
            for (int k = 0; k < 2; k++) {
                int kk = k ? Z.cp : Z.c0, km = k ? Z.c0 : Z.cm, kp = k ? Z.cpp : Z.cp;
                float t[3][8];
                if (fold) hcoef_p_unscaled<VARIANT>(m, ii, jj, kk, t);
                else hcoef_p<VARIANT>(m, ii, jj, kk, im, ip, jm, jp, km, kp, t);
#pragma unroll
                for (int c = 0; c < 3; c++)
#pragma unroll
                    for (int a = 0; a < 2; a++) {
                        float P0 = Z.f[k] * t[c][a * 4 + 0] + Z.g[k] * t[c][a * 4 + 1];
                        float P1 = Z.f[k] * t[c][a * 4 + 2] + Z.g[k] * t[c][a * 4 + 3];
                        Ax[c][a] += Y.f[j] * P0 + Y.g[j] * P1;
                        if (GY) Bx[c][a] += Y.df[j] * P0 + Y.dg[j] * P1;
                        if (GZ) {
                            float dP0 = Z.df[k] * t[c][a * 4 + 0] + Z.dg[k] * t[c][a * 4 + 1];
                            float dP1 = Z.df[k] * t[c][a * 4 + 2] + Z.dg[k] * t[c][a * 4 + 3];
                            dAx[c][a] += Y.f[j] * dP0 + Y.g[j] * dP1;
                        }
                    }
            }
        }
#pragma unroll
        for (int c = 0; c < 3; c++) {
            v[c] += X.f[i] * Ax[c][0] + X.g[i] * Ax[c][1];
            if (GX) gx[c] += X.df[i] * Ax[c][0] + X.dg[i] * Ax[c][1];
            if (GY) gy[c] += X.f[i] * Bx[c][0] + X.g[i] * Bx[c][1];
            if (GZ) gz[c] += X.f[i] * dAx[c][0] + X.g[i] * dAx[c][1];
        }
    }
    const float inv = 1.0f / m.dx;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        val[c] = v[c];
        if (GX) grad[c][0] = gx[c] * inv;
        if (GY) grad[c][1] = gy[c] * inv;
        if (GZ) grad[c][2] = gz[c] * inv;
    }
}

// ---------------------------------------------------------------------------
// RK4 marches (hermite.py:786-860, run_edge.py:337-357)
// ---------------------------------------------------------------------------
EDGE_D void rk4_pos(const Mac& mac, float psi[3], float dt) {
    float u1[3], u2[3], u3[3], u4[3], q[3];
    float h = 0.5f * dt;
    mac_sample<false>(mac, psi, u1, nullptr);
#pragma unroll
    for (int c = 0; c < 3; c++) q[c] = psi[c] + h * u1[c];
    mac_sample<false>(mac, q, u2, nullptr);
#pragma unroll
    for (int c = 0; c < 3; c++) q[c] = psi[c] + h * u2[c];
    mac_sample<false>(mac, q, u3, nullptr);
#pragma unroll
    for (int c = 0; c < 3; c++) q[c] = psi[c] + dt * u3[c];
    mac_sample<false>(mac, q, u4, nullptr);
    float w6 = dt * 1.0f / 6.0f;
#pragma unroll
    for (int c = 0; c < 3; c++) psi[c] = psi[c] + w6 * (u1[c] + 2.0f * u2[c] + 2.0f * u3[c] + u4[c]);
}

// RK4 of a point with NC Jacobian columns C[a] (dC/dt = grad u . C).  The
// four stages run as a loop (not unrolled): one copy of the 81-tap sampler
// keeps the kernels inside the instruction cache.
template <int NC>
EDGE_D void rk4_jac(const Mac& mac, float psi[3], float C[NC][3], float dt) {
    float u[3], G[3][3], q[3], Cs[NC][3], d[NC][3], su[3] = {0.0f, 0.0f, 0.0f}, sd[NC][3];
    float h = 0.5f * dt;
#pragma unroll
    for (int a = 0; a < NC; a++)
#pragma unroll
        for (int c = 0; c < 3; c++) sd[a][c] = 0.0f;
#pragma unroll
    for (int c = 0; c < 3; c++) q[c] = psi[c];
#pragma unroll
    for (int a = 0; a < NC; a++)
#pragma unroll
        for (int c = 0; c < 3; c++) Cs[a][c] = C[a][c];
#pragma unroll 1
    for (int stage = 0; stage < 4; stage++) {
        mac_sample<true>(mac, q, u, G);
        // derivative of the columns at this stage
#pragma unroll
        for (int a = 0; a < NC; a++)
#pragma unroll
            for (int r = 0; r < 3; r++) d[a][r] = G[r][0] * Cs[a][0] + G[r][1] * Cs[a][1] + G[r][2] * Cs[a][2];
        // the RK4 sums, started at zero: 0 + 1 * u is u exactly
        const float wt = (stage == 0 || stage == 3) ? 1.0f : 2.0f;
#pragma unroll
        for (int c = 0; c < 3; c++) su[c] = su[c] + wt * u[c];
#pragma unroll
        for (int a = 0; a < NC; a++)
#pragma unroll
            for (int c = 0; c < 3; c++) sd[a][c] = sd[a][c] + wt * d[a][c];
        if (stage < 3) {
            const float hh = stage < 2 ? h : dt;
#pragma unroll
            for (int c = 0; c < 3; c++) q[c] = psi[c] + hh * u[c];
#pragma unroll
            for (int a = 0; a < NC; a++)
#pragma unroll
                for (int c = 0; c < 3; c++) Cs[a][c] = C[a][c] + hh * d[a][c];
        }
    }
    float w6 = dt * 1.0f / 6.0f;
#pragma unroll
    for (int c = 0; c < 3; c++) psi[c] = psi[c] + w6 * su[c];
#pragma unroll
    for (int a = 0; a < NC; a++)
#pragma unroll
        for (int c = 0; c < 3; c++) C[a][c] = C[a][c] + w6 * sd[a][c];
}

EDGE_D void cell_pos(int i, int j, int k, float dx, float X[3]) {
    X[0] = ((float)i + 0.5f) * dx;
    X[1] = ((float)j + 0.5f) * dx;
    X[2] = ((float)k + 0.5f) * dx;
}
EDGE_D void face_pos(int axis, int i, int j, int k, float dx, float X[3]) {
    X[0] = ((float)i + (axis == 0 ? 0.0f : 0.5f)) * dx;
    X[1] = ((float)j + (axis == 1 ? 0.0f : 0.5f)) * dx;
    X[2] = ((float)k + (axis == 2 ? 0.0f : 0.5f)) * dx;
}

// Decompose a linear face index over the three face grids (x faces first).
struct FaceIdx {
    int axis, i, j, k, e;
};
EDGE_D FaceIdx face_decompose(long long t, int nx, int ny, int nz) {
    FaceIdx f;
    long long nfx = (long long)(nx + 1) * ny * nz, nfy = (long long)nx * (ny + 1) * nz;
    int n1, n2;
    if (t < nfx) { f.axis = 0; n1 = ny; n2 = nz; }
    else if (t < nfx + nfy) { f.axis = 1; t -= nfx; n1 = ny + 1; n2 = nz; }
    else { f.axis = 2; t -= nfx + nfy; n1 = ny; n2 = nz + 1; }
    // within one face grid the index fits 32 bits (f.e is an int): unsigned
    // 32-bit division instead of the 64-bit one
    const unsigned u = (unsigned)t;
    f.e = (int)u;
    f.k = (int)(u % (unsigned)n2);
    const unsigned r = u / (unsigned)n2;
    f.j = (int)(r % (unsigned)n1);
    f.i = (int)(r / (unsigned)n1);
    return f;
}

EDGE_HD long long n_faces(int nx, int ny, int nz) {
    return (long long)(nx + 1) * ny * nz + (long long)nx * (ny + 1) * nz + (long long)nx * ny * (nz + 1);
}

}  // namespace edge
