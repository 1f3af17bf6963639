// Flow-map marches, velocity / dye transport and point samplers of the EDGE
// step (sim/hermite.py, run_edge.py, run_ed4.py, run_ed8.py,
// util/taichi_utils.py), one thread per cell or face.
#include <cuda_runtime.h>
#include <cstdlib>

#include <algorithm>

#include "edge_common.cuh"

using namespace edge;

namespace {

constexpr int kBlock = 256;

inline int grid_for(long long n, int block = kBlock) { return (int)((n + block - 1) / block); }

inline int launch_status() {
    cudaError_t e = cudaPeekAtLastError();
    return e == cudaSuccess ? EDGE_OK : (int)e;
}

inline bool dims_ok(int nx, int ny, int nz) {
    if (nx < 4 || ny < 4 || nz < 4) return false;
    long long nf = n_faces(nx, ny, nz) * 3;  // vec3 face fields must index in int32
    long long nc4 = (long long)nx * ny * nz * 4;
    return nf < (1LL << 31) && nc4 < (1LL << 31);
}

inline bool al16(const void* p) { return p == nullptr || ((uintptr_t)p & 15) == 0; }

// ---------------------------------------------------------------------------
// point samplers
// ---------------------------------------------------------------------------
__global__ void k_points_mac(Mac mac, const float* __restrict__ pts, int n, float* v, float* vg, float* g) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    float p[3] = {pts[3 * e], pts[3 * e + 1], pts[3 * e + 2]};
    float a[3], b[3], G[3][3];
    mac_sample<false>(mac, p, a, nullptr);
    mac_sample<true>(mac, p, b, G);
    for (int c = 0; c < 3; c++) {
        v[3 * e + c] = a[c];
        vg[3 * e + c] = b[c];
        for (int d = 0; d < 3; d++) g[9 * e + 3 * c + d] = G[c][d];
    }
}

__global__ void k_points_dye(Dye dye, const float* __restrict__ smoke, const float* __restrict__ pts, int n,
                             float4* lin, float4* mn, float4* mx) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    float p[3] = {pts[3 * e], pts[3 * e + 1], pts[3 * e + 2]};
    Lin8 L = lin_setup(dye, p);
    lin[e] = dye_interp(smoke, dye, L);
    float4 a, b;
    dye_minmax(smoke, dye, L, a, b);
    mn[e] = a;
    mx[e] = b;
}

template <int V>
__global__ void k_points_hermite(MapF m, const float* __restrict__ pts, int n, float* val, float* gval,
                                 float* grad) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    float p[3] = {pts[3 * e], pts[3 * e + 1], pts[3 * e + 2]};
    float a[3], b[3], G[3][3];
    hermite3<V, false>(m, p, a, nullptr);
    hermite3<V, true>(m, p, b, G);
    for (int c = 0; c < 3; c++) {
        val[3 * e + c] = a[c];
        gval[3 * e + c] = b[c];
        for (int d = 0; d < 3; d++) grad[9 * e + 3 * c + d] = G[c][d];
    }
}

// ---------------------------------------------------------------------------
// resets (hermite.py:642-700, run_edge.py:306-320)
// ---------------------------------------------------------------------------
__global__ void k_reset_cells(int nx, int ny, int nz, float dx, float* psi, float* Tx, float* Ty, float* Tz,
                              float* dTx, float* dTy, float* dTz, float* d2Tx, float* d2Ty, float* d2Tz) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    int n = nx * ny * nz;
    if (e >= n) return;
    int k = e % nz, j = (e / nz) % ny, i = e / (ny * nz);
    float X[3];
    cell_pos(i, j, k, dx, X);
    float* T[3] = {Tx, Ty, Tz};
    float* dT[3] = {dTx, dTy, dTz};
    float* d2T[3] = {d2Tx, d2Ty, d2Tz};
    for (int c = 0; c < 3; c++) {
        psi[3 * e + c] = X[c];
        for (int d = 0; d < 3; d++) {
            T[c][3 * e + d] = c == d ? 1.0f : 0.0f;
            if (dT[c]) dT[c][3 * e + d] = 0.0f;
        }
        if (d2T[c]) d2T[c][e] = 0.0f;
    }
}

__global__ void k_reset_faces(int nx, int ny, int nz, float dx, float* phix, float* phiy, float* phiz, float* Fx,
                              float* Fy, float* Fz) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_faces(nx, ny, nz)) return;
    FaceIdx f = face_decompose(t, nx, ny, nz);
    float X[3];
    face_pos(f.axis, f.i, f.j, f.k, dx, X);
    float* phi = f.axis == 0 ? phix : (f.axis == 1 ? phiy : phiz);
    float* F = f.axis == 0 ? Fx : (f.axis == 1 ? Fy : Fz);
    for (int c = 0; c < 3; c++) {
        phi[3 * f.e + c] = X[c];
        F[3 * f.e + c] = c == f.axis ? 1.0f : 0.0f;
    }
}

// ---------------------------------------------------------------------------
// EDGE march (hermite.py:1426-1521)
// ---------------------------------------------------------------------------
__constant__ float c_ed4_off[4][3] = {{-1, -1, -1}, {1, 1, -1}, {-1, 1, 1}, {1, -1, 1}};    // hermite.py:1446-1449
__constant__ float c_ed8_off[8][3] = {{-1, -1, -1}, {1, -1, -1}, {-1, 1, -1}, {1, 1, -1},   // hermite.py:716-723
                                      {-1, -1, 1},  {1, -1, 1},  {-1, 1, 1},  {1, 1, 1}};

template <bool IDENT>
__global__ void __launch_bounds__(128) k_march_edge(Mac mac, MapF m, float dt, float eps, float* __restrict__ opsi,
                                                    float* __restrict__ oTx, float* __restrict__ oTy,
                                                    float* __restrict__ oTz, float* __restrict__ odTx,
                                                    float* __restrict__ odTy, float* __restrict__ odTz) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    int n = m.nx * m.ny * m.nz;
    if (e >= n) return;
    int k = e % m.nz, j = (e / m.nz) % m.ny, i = e / (m.ny * m.nz);
    float X[3];
    cell_pos(i, j, k, m.dx, X);
    // calc_ed4_garm_func (hermite.py:1049-1075) accumulated per point: A and B
    // groups of each mixed derivative, summed in the reference's order.
    float dA[3][3], dB[3][3];
    float Pc[3], Tc[3][3];
#pragma unroll 1
    for (int q = 0; q < 5; q++) {
        float P[3], C[3][3];
        for (int c = 0; c < 3; c++) {
            P[c] = q == 0 ? X[c] : X[c] + c_ed4_off[q - 1][c] * eps;
            for (int d = 0; d < 3; d++) C[c][d] = c == d ? 1.0f : 0.0f;  // columns of the identity
        }
        rk4_jac<3>(mac, P, C, -dt);
        float T[3][3];  // rows of the composed Jacobian
        if (IDENT) {
            // Hermite of the identity map reproduces the (clamped) position;
            // its gradient is the identity.
            for (int c = 0; c < 3; c++) {
                float u = over_dx(P[c], m.dx, m.inv_dx, m.pow2) - 0.5f;
                float s = fmaxf(1.0f, fminf(u, m.hi[c]));
                P[c] = (s + 0.5f) * m.dx;
                for (int d = 0; d < 3; d++) T[c][d] = C[d][c];
            }
        } else {
            float val[3], G[3][3];
            hermite3<HV_GARM, true>(m, P, val, G);
            // T = T_old @ T_step, T_step rows: T_step[r][d] = C[d][r]
            for (int r = 0; r < 3; r++)
                for (int d = 0; d < 3; d++) T[r][d] = G[r][0] * C[d][0] + G[r][1] * C[d][1] + G[r][2] * C[d][2];
            for (int c = 0; c < 3; c++) P[c] = val[c];
        }
        if (q == 0) {
            for (int c = 0; c < 3; c++) {
                Pc[c] = P[c];
                for (int d = 0; d < 3; d++) Tc[c][d] = T[c][d];
            }
        } else {
            float sx = c_ed4_off[q - 1][0], sy = c_ed4_off[q - 1][1], sz = c_ed4_off[q - 1][2];
            for (int c = 0; c < 3; c++) {
                float a0 = sz * T[c][1], b0 = sy * T[c][2];
                float a1 = sz * T[c][0], b1 = sx * T[c][2];
                float a2 = sy * T[c][0], b2 = sx * T[c][1];
                if (q == 1) {
                    dA[c][0] = a0; dB[c][0] = b0; dA[c][1] = a1; dB[c][1] = b1; dA[c][2] = a2; dB[c][2] = b2;
                } else {
                    dA[c][0] += a0; dB[c][0] += b0; dA[c][1] += a1; dB[c][1] += b1; dA[c][2] += a2; dB[c][2] += b2;
                }
            }
        }
    }
    float* oT[3] = {oTx, oTy, oTz};
    float* odT[3] = {odTx, odTy, odTz};
    for (int c = 0; c < 3; c++) {
        opsi[3 * e + c] = Pc[c];
        for (int d = 0; d < 3; d++) {
            oT[c][3 * e + d] = Tc[c][d];
            odT[c][3 * e + d] = (dA[c][d] + dB[c][d]) / 8.0f / eps;
        }
    }
}

// EDGE march on the packed layout (same algorithm as k_march_edge); output
// planes 0-6 of `out` (n cells per plane).
// T = T_old @ T_step (interp_psi_hermite_garm_fd_unroll_func,
// hermite.py:960-980) with T_step[a][d] = C[d][a]: float32 products and sums
// as the reference forms them, or (F64) each entry accumulated in float64 and
// rounded once
template <bool F64>
EDGE_D void compose_jac(const float (&G)[3][3], const float (&C)[3][3], float (&T)[3][3]) {
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int d = 0; d < 3; d++) {
            if (F64)
                T[r][d] = (float)fma((double)G[r][2], (double)C[d][2],
                                     fma((double)G[r][1], (double)C[d][1], (double)G[r][0] * (double)C[d][0]));
            else
                T[r][d] = G[r][0] * C[d][0] + G[r][1] * C[d][1] + G[r][2] * C[d][2];
        }
}

template <bool IDENT, bool F64, bool P2>
__global__ void __launch_bounds__(128, 5) k_march_edge_p(Mac mac_, MapP m_, float dt, float eps, float4* __restrict__ out) {
    const Mac mac = with_pow2<P2>(mac_);
    const MapP m = with_pow2<P2>(m_);
    // The per-cell accumulators (the centre point's psi and Jacobian, the A
    // and B groups of the mixed derivatives) live in shared memory, one
    // column per thread, so that the registers hold only the current
    // point's trajectory: 5 blocks of 128 threads per SM (96 registers)
    // instead of 3 (168): march at 256x128x128 4.14 -> 3.80 ms (4 blocks:
    // 3.97 ms).
    __shared__ float acc[30][128];
    float(&Pc)[3][128] = *reinterpret_cast<float(*)[3][128]>(&acc[0][0]);
    float(&Tc)[9][128] = *reinterpret_cast<float(*)[9][128]>(&acc[3][0]);
    float(&dA)[9][128] = *reinterpret_cast<float(*)[9][128]>(&acc[12][0]);
    float(&dB)[9][128] = *reinterpret_cast<float(*)[9][128]>(&acc[21][0]);
    const int tx = threadIdx.x;
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = m.n;
    if (e >= n) return;
    int k = e % m.nz, j = (e / m.nz) % m.ny, i = e / (m.ny * m.nz);
    float X[3];
    cell_pos(i, j, k, m.dx, X);
#pragma unroll 1
    for (int q = 0; q < 5; q++) {
        float P[3], C[3][3];
        for (int c = 0; c < 3; c++) {
            P[c] = q == 0 ? X[c] : X[c] + c_ed4_off[q - 1][c] * eps;
            for (int d = 0; d < 3; d++) C[c][d] = c == d ? 1.0f : 0.0f;
        }
        rk4_jac<3>(mac, P, C, -dt);
        float T[3][3];
        if (IDENT) {
            for (int c = 0; c < 3; c++) {
                float u = over_dx(P[c], m.dx, m.inv_dx, m.pow2) - 0.5f;
                float s = fmaxf(1.0f, fminf(u, m.hi[c]));
                P[c] = (s + 0.5f) * m.dx;
                for (int d = 0; d < 3; d++) T[c][d] = C[d][c];
            }
        } else {
            float val[3], G[3][3];
            hermite3p<HV_GARM_P, true>(m, P, val, G);
            compose_jac<F64>(G, C, T);
            for (int c = 0; c < 3; c++) P[c] = val[c];
        }
        if (q == 0) {
            for (int c = 0; c < 3; c++) {
                Pc[c][tx] = P[c];
                for (int d = 0; d < 3; d++) Tc[3 * c + d][tx] = T[c][d];
            }
        } else {
            float sx = c_ed4_off[q - 1][0], sy = c_ed4_off[q - 1][1], sz = c_ed4_off[q - 1][2];
            for (int c = 0; c < 3; c++) {
                float a0 = sz * T[c][1], b0 = sy * T[c][2];
                float a1 = sz * T[c][0], b1 = sx * T[c][2];
                float a2 = sy * T[c][0], b2 = sx * T[c][1];
                if (q == 1) {
                    dA[3 * c][tx] = a0; dB[3 * c][tx] = b0; dA[3 * c + 1][tx] = a1; dB[3 * c + 1][tx] = b1;
                    dA[3 * c + 2][tx] = a2; dB[3 * c + 2][tx] = b2;
                } else {
                    dA[3 * c][tx] += a0; dB[3 * c][tx] += b0; dA[3 * c + 1][tx] += a1; dB[3 * c + 1][tx] += b1;
                    dA[3 * c + 2][tx] += a2; dB[3 * c + 2][tx] += b2;
                }
            }
        }
    }
    out[e] = make_float4(Pc[0][tx], Pc[1][tx], Pc[2][tx], 0.f);
#pragma unroll
    for (int d = 0; d < 3; d++) {
        out[(size_t)(1 + d) * n + e] = make_float4(Tc[d][tx], Tc[3 + d][tx], Tc[6 + d][tx], 0.f);
        out[(size_t)(4 + d) * n + e] =
            make_float4((dA[d][tx] + dB[d][tx]) / 8.0f / eps, (dA[3 + d][tx] + dB[3 + d][tx]) / 8.0f / eps,
                        (dA[6 + d][tx] + dB[6 + d][tx]) / 8.0f / eps, 0.f);
    }
}

// ED4 march on the packed layout; output planes 0-3.
template <bool P2>
__global__ void __launch_bounds__(128) k_march_ed4_p(Mac mac_, MapP m_, float dt, float eps, float4* __restrict__ out) {
    const Mac mac = with_pow2<P2>(mac_);
    const MapP m = with_pow2<P2>(m_);
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = m.n;
    if (e >= n) return;
    int k = e % m.nz, j = (e / m.nz) % m.ny, i = e / (m.ny * m.nz);
    float X[3];
    cell_pos(i, j, k, m.dx, X);
    float P[4][3];
#pragma unroll 1
    for (int q = 0; q < 4; q++) {
        float p[3];
        for (int c = 0; c < 3; c++) p[c] = X[c] + c_ed4_off[q][c] * eps;
        rk4_pos(mac, p, -dt);
        float v[3];
        hermite3p<HV_FD_P, false>(m, p, v, nullptr);
        for (int c = 0; c < 3; c++) P[q][c] = v[c];
    }
    float o[4][3];
    for (int c = 0; c < 3; c++) {
        o[0][c] = (P[0][c] + P[1][c] + P[2][c] + P[3][c]) / 4.0f;
        o[1][c] = (-P[0][c] + P[1][c] - P[2][c] + P[3][c]) / 4.0f / eps;
        o[2][c] = (-P[0][c] + P[1][c] + P[2][c] - P[3][c]) / 4.0f / eps;
        o[3][c] = (-P[0][c] - P[1][c] + P[2][c] + P[3][c]) / 4.0f / eps;
    }
    for (int q = 0; q < 4; q++) out[(size_t)q * n + e] = make_float4(o[q][0], o[q][1], o[q][2], 0.f);
}

// ED8 march on the packed layout; output planes 0-7.
template <bool P2>
__global__ void __launch_bounds__(128) k_march_ed8_p(Mac mac_, MapP m_, float dt, float eps, float4* __restrict__ out) {
    const Mac mac = with_pow2<P2>(mac_);
    const MapP m = with_pow2<P2>(m_);
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = m.n;
    if (e >= n) return;
    int k = e % m.nz, j = (e / m.nz) % m.ny, i = e / (m.ny * m.nz);
    float X[3];
    cell_pos(i, j, k, m.dx, X);
    float P[8][3];
#pragma unroll 1
    for (int q = 0; q < 8; q++) {
        float p[3];
        for (int c = 0; c < 3; c++) p[c] = X[c] + c_ed8_off[q][c] * eps;
        rk4_pos(mac, p, -dt);
        float v[3];
        hermite3p<HV_FULL, false>(m, p, v, nullptr);
        for (int c = 0; c < 3; c++) P[q][c] = v[c];
    }
    float o[8][3];
    for (int c = 0; c < 3; c++) {
        float a0 = P[0][c], a1 = P[1][c], a2 = P[2][c], a3 = P[3][c];
        float a4 = P[4][c], a5 = P[5][c], a6 = P[6][c], a7 = P[7][c];
        o[0][c] = (a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7) / 8.0f;
        o[1][c] = (-a0 + a1 - a2 + a3 - a4 + a5 - a6 + a7) / 8.0f / eps;
        o[2][c] = (-a0 - a1 + a2 + a3 - a4 - a5 + a6 + a7) / 8.0f / eps;
        o[3][c] = (-a0 - a1 - a2 - a3 + a4 + a5 + a6 + a7) / 8.0f / eps;
        o[4][c] = (a0 + a1 - a2 - a3 - a4 - a5 + a6 + a7) / 8.0f / eps / eps;
        o[5][c] = (a0 - a1 + a2 - a3 - a4 + a5 - a6 + a7) / 8.0f / eps / eps;
        o[6][c] = (a0 - a1 - a2 + a3 + a4 - a5 - a6 + a7) / 8.0f / eps / eps;
        o[7][c] = (-a0 + a1 + a2 - a3 + a4 - a5 - a6 + a7) / 8.0f / eps / eps / eps;
    }
    for (int q = 0; q < 8; q++) out[(size_t)q * n + e] = make_float4(o[q][0], o[q][1], o[q][2], 0.f);
}

// GE march (hermite.py:1398-1424 advect_ps_garm up to its copies): the cell
// centre is marched back by RK4 with its Jacobian from the identity
// (hermite.py:643-654, 864-918 with -dt) and composed with the accumulated
// map through the full stored-derivative Hermite (hermite.py:1024-1046).
// dT and d2T of the new map come from calc_fd_3_from_grad afterwards.
EDGE_D void herm_full(const MapF& m, const float p[3], float v[3], float g[3][3]) { hermite3<HV_FULL, true>(m, p, v, g); }
EDGE_D void herm_full(const MapP& m, const float p[3], float v[3], float g[3][3]) { hermite3p<HV_FULL, true>(m, p, v, g); }

template <class M, bool F64 = false>
EDGE_D void ge_center(const Mac& mac, const M& m, int e, float dt, float P[3], float (&T)[3][3]) {
    int k = e % m.nz, j = (e / m.nz) % m.ny, i = e / (m.ny * m.nz);
    cell_pos(i, j, k, m.dx, P);
    float C[3][3];
    for (int c = 0; c < 3; c++)
        for (int d = 0; d < 3; d++) C[c][d] = c == d ? 1.0f : 0.0f;
    rk4_jac<3>(mac, P, C, -dt);
    float val[3], G[3][3];
    herm_full(m, P, val, G);
    compose_jac<F64>(G, C, T);  // T = T_old @ T_step
    for (int c = 0; c < 3; c++) P[c] = val[c];
}

__global__ void __launch_bounds__(128) k_march_ge(Mac mac, MapF m, float dt, float* __restrict__ opsi,
                                                  float* __restrict__ oTx, float* __restrict__ oTy,
                                                  float* __restrict__ oTz) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.nx * m.ny * m.nz) return;
    float P[3], T[3][3];
    ge_center(mac, m, e, dt, P, T);
    float* oT[3] = {oTx, oTy, oTz};
    for (int c = 0; c < 3; c++) {
        opsi[3 * e + c] = P[c];
        for (int d = 0; d < 3; d++) oT[c][3 * e + d] = T[c][d];
    }
}

// packed layout: planes 0-3 of `out`
template <bool F64, bool P2>
__global__ void __launch_bounds__(128) k_march_ge_p(Mac mac_, MapP m_, float dt, float4* __restrict__ out) {
    const Mac mac = with_pow2<P2>(mac_);
    const MapP m = with_pow2<P2>(m_);
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = m.n;
    if (e >= n) return;
    float P[3], T[3][3];
    ge_center<MapP, F64>(mac, m, e, dt, P, T);
    out[e] = make_float4(P[0], P[1], P[2], 0.f);
#pragma unroll
    for (int d = 0; d < 3; d++) out[(size_t)(1 + d) * n + e] = make_float4(T[0][d], T[1][d], T[2][d], 0.f);
}

// calc_fd_3_from_grad (hermite.py:1180-1256), first loops: dT_c from central
// differences of the gradient row T_c, neighbour index clamped to the grid.
// One thread per cell and component.
__global__ void k_fd3_dT(int nx, int ny, int nz, float dx, const float* __restrict__ Tx,
                         const float* __restrict__ Ty, const float* __restrict__ Tz, float* dTx, float* dTy,
                         float* dTz) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int n = nx * ny * nz;
    if (t >= 3LL * n) return;
    const int c = (int)(t / n), e = (int)(t - (long long)c * n);
    const float* T = c == 0 ? Tx : (c == 1 ? Ty : Tz);
    float* o = c == 0 ? dTx : (c == 1 ? dTy : dTz);
    const int k = e % nz, j = (e / nz) % ny, i = e / (ny * nz);
    const int ip = min(i + 1, nx - 1), im = max(i - 1, 0), jp = min(j + 1, ny - 1), jm = max(j - 1, 0);
    const int kp = min(k + 1, nz - 1), km = max(k - 1, 0);
    const float* Tkp = T + 3 * idx3(i, j, kp, ny, nz);
    const float* Tkm = T + 3 * idx3(i, j, km, ny, nz);
    const float* Tjp = T + 3 * idx3(i, jp, k, ny, nz);
    const float* Tjm = T + 3 * idx3(i, jm, k, ny, nz);
    const float* Tip = T + 3 * idx3(ip, j, k, ny, nz);
    const float* Tim = T + 3 * idx3(im, j, k, ny, nz);
    o[3 * e + 0] = ((__ldg(Tkp + 1) - __ldg(Tkm + 1)) + (__ldg(Tjp + 2) - __ldg(Tjm + 2))) / 4.0f / dx;
    o[3 * e + 1] = ((__ldg(Tkp + 0) - __ldg(Tkm + 0)) + (__ldg(Tip + 2) - __ldg(Tim + 2))) / 4.0f / dx;
    o[3 * e + 2] = ((__ldg(Tjp + 0) - __ldg(Tjm + 0)) + (__ldg(Tip + 1) - __ldg(Tim + 1))) / 4.0f / dx;
}

// calc_fd_3_from_grad, last loops: d2T_c from central differences of dT_c.
__global__ void k_fd3_d2T(int nx, int ny, int nz, float dx, const float* __restrict__ dTx,
                          const float* __restrict__ dTy, const float* __restrict__ dTz, float* d2Tx, float* d2Ty,
                          float* d2Tz) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int n = nx * ny * nz;
    if (t >= 3LL * n) return;
    const int c = (int)(t / n), e = (int)(t - (long long)c * n);
    const float* D = c == 0 ? dTx : (c == 1 ? dTy : dTz);
    float* o = c == 0 ? d2Tx : (c == 1 ? d2Ty : d2Tz);
    const int k = e % nz, j = (e / nz) % ny, i = e / (ny * nz);
    const int ip = min(i + 1, nx - 1), im = max(i - 1, 0), jp = min(j + 1, ny - 1), jm = max(j - 1, 0);
    const int kp = min(k + 1, nz - 1), km = max(k - 1, 0);
    o[e] = ((__ldg(D + 3 * idx3(ip, j, k, ny, nz)) - __ldg(D + 3 * idx3(im, j, k, ny, nz))) +
            (__ldg(D + 3 * idx3(i, jp, k, ny, nz) + 1) - __ldg(D + 3 * idx3(i, jm, k, ny, nz) + 1)) +
            (__ldg(D + 3 * idx3(i, j, kp, ny, nz) + 2) - __ldg(D + 3 * idx3(i, j, km, ny, nz) + 2))) /
           6.0f / dx;
}

// The same two passes on the packed planes: plane 1+d holds column d of the
// gradient (component c = psi_c,d), plane 4+d the mixed derivative dT_c[d]
// and plane 7 d2T_c, so every difference runs on the three components at once.
EDGE_D float4 f4sub(float4 a, float4 b) { return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, 0.f); }
EDGE_D float4 f4add(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, 0.f); }
EDGE_D float4 f4div(float4 a, float s, float dx) {
    return make_float4(a.x / s / dx, a.y / s / dx, a.z / s / dx, 0.f);
}

__global__ void k_fd3_dT_p(int nx, int ny, int nz, float dx, float4* __restrict__ g) {
    const int n = nx * ny * nz;
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const int k = e % nz, j = (e / nz) % ny, i = e / (ny * nz);
    const int ekp = idx3(i, j, min(k + 1, nz - 1), ny, nz), ekm = idx3(i, j, max(k - 1, 0), ny, nz);
    const int ejp = idx3(i, min(j + 1, ny - 1), k, ny, nz), ejm = idx3(i, max(j - 1, 0), k, ny, nz);
    const int eip = idx3(min(i + 1, nx - 1), j, k, ny, nz), eim = idx3(max(i - 1, 0), j, k, ny, nz);
    const float4* P1 = g + (size_t)1 * n;
    const float4* P2 = g + (size_t)2 * n;
    const float4* P3 = g + (size_t)3 * n;
    float4 yz = f4add(f4sub(__ldg(P2 + ekp), __ldg(P2 + ekm)), f4sub(__ldg(P3 + ejp), __ldg(P3 + ejm)));
    float4 xz = f4add(f4sub(__ldg(P1 + ekp), __ldg(P1 + ekm)), f4sub(__ldg(P3 + eip), __ldg(P3 + eim)));
    float4 xy = f4add(f4sub(__ldg(P1 + ejp), __ldg(P1 + ejm)), f4sub(__ldg(P2 + eip), __ldg(P2 + eim)));
    g[(size_t)4 * n + e] = f4div(yz, 4.0f, dx);
    g[(size_t)5 * n + e] = f4div(xz, 4.0f, dx);
    g[(size_t)6 * n + e] = f4div(xy, 4.0f, dx);
}

__global__ void k_fd3_d2T_p(int nx, int ny, int nz, float dx, float4* __restrict__ g) {
    const int n = nx * ny * nz;
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const int k = e % nz, j = (e / nz) % ny, i = e / (ny * nz);
    const float4* P4 = g + (size_t)4 * n;
    const float4* P5 = g + (size_t)5 * n;
    const float4* P6 = g + (size_t)6 * n;
    float4 s = f4add(f4add(f4sub(__ldg(P4 + idx3(min(i + 1, nx - 1), j, k, ny, nz)),
                                 __ldg(P4 + idx3(max(i - 1, 0), j, k, ny, nz))),
                           f4sub(__ldg(P5 + idx3(i, min(j + 1, ny - 1), k, ny, nz)),
                                 __ldg(P5 + idx3(i, max(j - 1, 0), k, ny, nz)))),
                     f4sub(__ldg(P6 + idx3(i, j, min(k + 1, nz - 1), ny, nz)),
                           __ldg(P6 + idx3(i, j, max(k - 1, 0), ny, nz))));
    g[(size_t)7 * n + e] = f4div(s, 6.0f, dx);
}

// The derived planes of a packed ED4 (V = HV_FD: planes 4-7) or EDGE
// (V = HV_GARM: plane 7) map: the finite-difference Hermite coefficients of
// each cell as a corner (hcoef_p's expressions with the cell's +-1 neighbours
// clamped to the grid), before their final multiplications by dx, which the
// evaluation applies; so they do not depend on dx and the evaluation's
// coefficients are bit for bit the ones hcoef_p forms.
template <int V>
__global__ void k_coef_p(MapP m, float4* __restrict__ g) {
    const int n = m.n, n1 = m.ny, n2 = m.nz;
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const int kk = e % m.nz, jj = (e / m.nz) % m.ny, ii = e / (m.ny * m.nz);
    const int im = max(ii - 1, 0), ip = min(ii + 1, m.nx - 1), jm = max(jj - 1, 0), jp = min(jj + 1, m.ny - 1);
    const int km = max(kk - 1, 0), kp = min(kk + 1, m.nz - 1);
    float o[4][3];
    if (V == HV_FD) {
        // hermite.py:104-148
        const int ekp = idx3(ii, jj, kp, n1, n2), ekm = idx3(ii, jj, km, n1, n2);
        const int ejp = idx3(ii, jp, kk, n1, n2), ejm = idx3(ii, jm, kk, n1, n2);
        const int eip = idx3(ip, jj, kk, n1, n2), eim = idx3(im, jj, kk, n1, n2);
        float4 kp1 = ldp(m, 2, ekp), km1 = ldp(m, 2, ekm), kp0 = ldp(m, 1, ekp), km0 = ldp(m, 1, ekm);
        float4 jp2 = ldp(m, 3, ejp), jm2 = ldp(m, 3, ejm), jp0 = ldp(m, 1, ejp), jm0 = ldp(m, 1, ejm);
        float4 ip2 = ldp(m, 3, eip), im2 = ldp(m, 3, eim), ip1 = ldp(m, 2, eip), im1 = ldp(m, 2, eim);
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
            o[0][c] = ((c4(kp1, c) - c4(km1, c)) + (c4(jp2, c) - c4(jm2, c))) / 4.0f;
            o[1][c] = ((c4(kp0, c) - c4(km0, c)) + (c4(ip2, c) - c4(im2, c))) / 4.0f;
            o[2][c] = ((c4(jp0, c) - c4(jm0, c)) + (c4(ip1, c) - c4(im1, c))) / 4.0f;
            float v30 = ((c4(a30, c) - c4(b30, c)) + (c4(c30, c) - c4(d30, c))) / 4.0f;
            float v31 = ((c4(a31, c) - c4(b31, c)) + (c4(c31, c) - c4(d31, c))) / 4.0f;
            float v32 = ((c4(a32, c) - c4(b32, c)) + (c4(c32, c) - c4(d32, c))) / 4.0f;
            float v33 = ((c4(a33, c) - c4(b33, c)) + (c4(c33, c) - c4(d33, c))) / 4.0f;
            float v34 = ((c4(a34, c) - c4(b34, c)) + (c4(c34, c) - c4(d34, c))) / 4.0f;
            float v35 = ((c4(a35, c) - c4(b35, c)) + (c4(c35, c) - c4(d35, c))) / 4.0f;
            o[3][c] = (v30 - v31 + v32 - v33 + v34 - v35) / 6.0f;
        }
        g[(size_t)4 * n + e] = make_float4(o[0][0], o[0][1], o[0][2], 0.f);
        g[(size_t)5 * n + e] = make_float4(o[1][0], o[1][1], o[1][2], 0.f);
        g[(size_t)6 * n + e] = make_float4(o[2][0], o[2][1], o[2][2], 0.f);
    } else {
        // hermite.py:346-351
        float4 xp = ldp(m, 4, idx3(ip, jj, kk, n1, n2)), xm = ldp(m, 4, idx3(im, jj, kk, n1, n2));
        float4 yp = ldp(m, 5, idx3(ii, jp, kk, n1, n2)), ym = ldp(m, 5, idx3(ii, jm, kk, n1, n2));
        float4 zp = ldp(m, 6, idx3(ii, jj, kp, n1, n2)), zm = ldp(m, 6, idx3(ii, jj, km, n1, n2));
#pragma unroll
        for (int c = 0; c < 3; c++)
            o[3][c] = ((c4(xp, c) - c4(xm, c)) + (c4(yp, c) - c4(ym, c)) + (c4(zp, c) - c4(zm, c))) / 6.0f;
    }
    g[(size_t)7 * n + e] = make_float4(o[3][0], o[3][1], o[3][2], 0.f);
}

// face map on the packed layout, one launch per face axis A: the map at the
// face and the derivative along A (only that gradient column is evaluated)
// (register caps: ED4 / EDGE 128 registers, 4 CTAs per SM; ED8 102, 5 CTAs
// per SM; both measured faster than the uncapped builds)
template <int V, int A, bool P2>
__global__ void __launch_bounds__(128, V == HV_FULL ? 5 : 4) k_face_map_p(MapP m_, float* fp, float* fc) {
    const MapP m = with_pow2<P2>(m_);
    const int n1 = m.ny + (A == 1), n2 = m.nz + (A == 2);
    const long long nf = (long long)(m.nx + (A == 0)) * n1 * n2;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nf) return;
    const unsigned u = (unsigned)t;  // one face grid: fits 32 bits
    const int e = (int)u;
    const int k = (int)(u % (unsigned)n2);
    const unsigned r = u / (unsigned)n2;
    const int j = (int)(r % (unsigned)n1), i = (int)(r / (unsigned)n1);
    float X[3], val[3], G[3][3];
    face_pos(A, i, j, k, m.dx, X);
    hermite3p<V, true, A>(m, X, val, G);
#pragma unroll
    for (int c = 0; c < 3; c++) {
        fp[3 * e + c] = val[c];
        fc[3 * e + c] = G[c][A];
    }
}

// reference layout (psi, T_c rows, dT_c, d2T_c) <-> packed planes
__global__ void k_map_pack(int n, int planes, const float* psi, const float* Tx, const float* Ty, const float* Tz,
                           const float* dTx, const float* dTy, const float* dTz, const float* d2x, const float* d2y,
                           const float* d2z, float4* out) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    out[e] = make_float4(psi[3 * e], psi[3 * e + 1], psi[3 * e + 2], 0.f);
    for (int d = 0; d < 3; d++)
        out[(size_t)(1 + d) * n + e] = make_float4(Tx[3 * e + d], Ty[3 * e + d], Tz[3 * e + d], 0.f);
    if (planes >= 7)
        for (int d = 0; d < 3; d++)
            out[(size_t)(4 + d) * n + e] = make_float4(dTx[3 * e + d], dTy[3 * e + d], dTz[3 * e + d], 0.f);
    if (planes >= 8) out[(size_t)7 * n + e] = make_float4(d2x[e], d2y[e], d2z[e], 0.f);
}

__global__ void k_map_unpack(int n, int planes, const float4* in, float* psi, float* Tx, float* Ty, float* Tz,
                             float* dTx, float* dTy, float* dTz, float* d2x, float* d2y, float* d2z) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    float4 v = in[e];
    psi[3 * e] = v.x; psi[3 * e + 1] = v.y; psi[3 * e + 2] = v.z;
    for (int d = 0; d < 3; d++) {
        float4 g = in[(size_t)(1 + d) * n + e];
        Tx[3 * e + d] = g.x; Ty[3 * e + d] = g.y; Tz[3 * e + d] = g.z;
    }
    if (planes >= 7)
        for (int d = 0; d < 3; d++) {
            float4 g = in[(size_t)(4 + d) * n + e];
            dTx[3 * e + d] = g.x; dTy[3 * e + d] = g.y; dTz[3 * e + d] = g.z;
        }
    if (planes >= 8) {
        float4 g = in[(size_t)7 * n + e];
        d2x[e] = g.x; d2y[e] = g.y; d2z[e] = g.z;
    }
}

// ED4 march (hermite.py:1375-1395): 4 epsilon points, RK4 of the position,
// FD-Hermite composition, calc_ed4_1 (hermite.py:1154-1177).
__global__ void __launch_bounds__(128) k_march_ed4(Mac mac, MapF m, float dt, float eps, float* __restrict__ opsi,
                                                   float* __restrict__ oTx, float* __restrict__ oTy,
                                                   float* __restrict__ oTz) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    int n = m.nx * m.ny * m.nz;
    if (e >= n) return;
    int k = e % m.nz, j = (e / m.nz) % m.ny, i = e / (m.ny * m.nz);
    float X[3];
    cell_pos(i, j, k, m.dx, X);
    float P[4][3];
#pragma unroll 1
    for (int q = 0; q < 4; q++) {
        float p[3];
        for (int c = 0; c < 3; c++) p[c] = X[c] + c_ed4_off[q][c] * eps;
        rk4_pos(mac, p, -dt);
        float v[3];
        hermite3<HV_FD, false>(m, p, v, nullptr);
        for (int c = 0; c < 3; c++) P[q][c] = v[c];
    }
    float* oT[3] = {oTx, oTy, oTz};
    for (int c = 0; c < 3; c++) {
        opsi[3 * e + c] = (P[0][c] + P[1][c] + P[2][c] + P[3][c]) / 4.0f;
        oT[c][3 * e + 0] = (-P[0][c] + P[1][c] - P[2][c] + P[3][c]) / 4.0f / eps;
        oT[c][3 * e + 1] = (-P[0][c] + P[1][c] + P[2][c] - P[3][c]) / 4.0f / eps;
        oT[c][3 * e + 2] = (-P[0][c] - P[1][c] + P[2][c] + P[3][c]) / 4.0f / eps;
    }
}

// ED8 march (hermite.py:1290-1338): 8 cube-corner points, full Hermite
// composition, calc_ed8_3 (hermite.py:1098-1151).
__global__ void __launch_bounds__(128) k_march_ed8(Mac mac, MapF m, float dt, float eps, float* __restrict__ opsi,
                                                   float* oTx, float* oTy, float* oTz, float* odTx, float* odTy,
                                                   float* odTz, float* od2Tx, float* od2Ty, float* od2Tz) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    int n = m.nx * m.ny * m.nz;
    if (e >= n) return;
    int k = e % m.nz, j = (e / m.nz) % m.ny, i = e / (m.ny * m.nz);
    float X[3];
    cell_pos(i, j, k, m.dx, X);
    float P[8][3];
#pragma unroll 1
    for (int q = 0; q < 8; q++) {
        float p[3];
        for (int c = 0; c < 3; c++) p[c] = X[c] + c_ed8_off[q][c] * eps;
        rk4_pos(mac, p, -dt);
        float v[3];
        hermite3<HV_FULL, false>(m, p, v, nullptr);
        for (int c = 0; c < 3; c++) P[q][c] = v[c];
    }
    float* oT[3] = {oTx, oTy, oTz};
    float* odT[3] = {odTx, odTy, odTz};
    float* od2T[3] = {od2Tx, od2Ty, od2Tz};
    for (int c = 0; c < 3; c++) {
        float a0 = P[0][c], a1 = P[1][c], a2 = P[2][c], a3 = P[3][c];
        float a4 = P[4][c], a5 = P[5][c], a6 = P[6][c], a7 = P[7][c];
        opsi[3 * e + c] = (a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7) / 8.0f;
        oT[c][3 * e + 0] = (-a0 + a1 - a2 + a3 - a4 + a5 - a6 + a7) / 8.0f / eps;
        oT[c][3 * e + 1] = (-a0 - a1 + a2 + a3 - a4 - a5 + a6 + a7) / 8.0f / eps;
        oT[c][3 * e + 2] = (-a0 - a1 - a2 - a3 + a4 + a5 + a6 + a7) / 8.0f / eps;
        odT[c][3 * e + 0] = (a0 + a1 - a2 - a3 - a4 - a5 + a6 + a7) / 8.0f / eps / eps;
        odT[c][3 * e + 1] = (a0 - a1 + a2 - a3 - a4 + a5 - a6 + a7) / 8.0f / eps / eps;
        odT[c][3 * e + 2] = (a0 - a1 - a2 + a3 + a4 - a5 - a6 + a7) / 8.0f / eps / eps;
        od2T[c][e] = (-a0 + a1 + a2 - a3 + a4 - a5 - a6 + a7) / 8.0f / eps / eps / eps;
    }
}

// Hermite psi and Jacobian column `axis` at every face (see edge_face_map).
template <int V>
__global__ void __launch_bounds__(128) k_face_map(MapF m, float* fpx, float* fpy, float* fpz, float* fcx,
                                                  float* fcy, float* fcz) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_faces(m.nx, m.ny, m.nz)) return;
    FaceIdx f = face_decompose(t, m.nx, m.ny, m.nz);
    float X[3], val[3], G[3][3];
    face_pos(f.axis, f.i, f.j, f.k, m.dx, X);
    hermite3<V, true>(m, X, val, G);
    float* fp = f.axis == 0 ? fpx : (f.axis == 1 ? fpy : fpz);
    float* fc = f.axis == 0 ? fcx : (f.axis == 1 ? fcy : fcz);
    for (int c = 0; c < 3; c++) {
        fp[3 * f.e + c] = val[c];
        fc[3 * f.e + c] = sel3(G[c], f.axis);
    }
}

// advance_map x3 (run_edge.py:330-357)
template <bool P2>
__global__ void __launch_bounds__(128) k_advance_map(Mac mac_, float dt, float* phix, float* phiy, float* phiz,
                                                     float* Fx, float* Fy, float* Fz) {
    const Mac mac = with_pow2<P2>(mac_);
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_faces(mac.nx, mac.ny, mac.nz)) return;
    FaceIdx f = face_decompose(t, mac.nx, mac.ny, mac.nz);
    float* phi = f.axis == 0 ? phix : (f.axis == 1 ? phiy : phiz);
    float* F = f.axis == 0 ? Fx : (f.axis == 1 ? Fy : Fz);
    float P[3], C[1][3];
    for (int c = 0; c < 3; c++) {
        P[c] = phi[3 * f.e + c];
        C[0][c] = F[3 * f.e + c];
    }
    rk4_jac<1>(mac, P, C, dt);
    for (int c = 0; c < 3; c++) {
        phi[3 * f.e + c] = P[c];
        F[3 * f.e + c] = C[0][c];
    }
}

// EFM backward map (run_efm.py:179-186 backtrack_psi_grid): every face starts
// at the identity (reset_to_identity, run_efm.py:153-167) and is marched by
// advance_map with -dts[s] through the cached velocities, newest first.  The
// reference runs one advance_map kernel per cached step and stores psi, T in
// between; here the whole chain runs in registers in one launch, so the map
// crosses HBM once (the float32 values between steps are the same).
constexpr int kMaxBacktrack = 64;
struct VelRing {
    const float* u[kMaxBacktrack][3];  // in application order (newest first)
    float dt[kMaxBacktrack];           // signed steps (-dts[s])
    int steps;
};

template <bool P2>
__global__ void __launch_bounds__(128) k_backtrack_faces(Mac mac_, VelRing ring, float* px, float* py, float* pz,
                                                         float* Tx, float* Ty, float* Tz) {
    const Mac mac = with_pow2<P2>(mac_);
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_faces(mac.nx, mac.ny, mac.nz)) return;
    FaceIdx f = face_decompose(t, mac.nx, mac.ny, mac.nz);
    float P[3], C[1][3];
    face_pos(f.axis, f.i, f.j, f.k, mac.dx, P);
    for (int c = 0; c < 3; c++) C[0][c] = c == f.axis ? 1.0f : 0.0f;
#pragma unroll 1
    for (int s = 0; s < ring.steps; s++) {
        Mac m = mac;
        m.u[0] = ring.u[s][0];
        m.u[1] = ring.u[s][1];
        m.u[2] = ring.u[s][2];
        rk4_jac<1>(m, P, C, ring.dt[s]);
    }
    float* p = f.axis == 0 ? px : (f.axis == 1 ? py : pz);
    float* T = f.axis == 0 ? Tx : (f.axis == 1 ? Ty : Tz);
    for (int c = 0; c < 3; c++) {
        p[3 * f.e + c] = P[c];
        T[3 * f.e + c] = C[0][c];
    }
}

// advect_u_semi_lagrangian (hermite.py:1578-1621)
template <bool P2>
__global__ void __launch_bounds__(128) k_advect_sl(Mac mac_, float dt, float* ox, float* oy, float* oz) {
    const Mac mac = with_pow2<P2>(mac_);
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_faces(mac.nx, mac.ny, mac.nz)) return;
    FaceIdx f = face_decompose(t, mac.nx, mac.ny, mac.nz);
    float p1[3], v1[3], v2[3], v3[3], v4[3], q[3];
    face_pos(f.axis, f.i, f.j, f.k, mac.dx, p1);
    mac_sample<false>(mac, p1, v1, nullptr);
    for (int c = 0; c < 3; c++) q[c] = p1[c] - v1[c] * dt * 0.5f;
    mac_sample<false>(mac, q, v2, nullptr);
    for (int c = 0; c < 3; c++) q[c] = p1[c] - v2[c] * dt * 0.5f;
    mac_sample<false>(mac, q, v3, nullptr);
    for (int c = 0; c < 3; c++) q[c] = p1[c] - v3[c] * dt;
    mac_sample<false>(mac, q, v4, nullptr);
    for (int c = 0; c < 3; c++) q[c] = p1[c] - (v1[c] + 2.0f * v2[c] + 2.0f * v3[c] + v4[c]) / 6.0f * dt;
    // only the face's own component of the last sample is kept
    float* o = f.axis == 0 ? ox : (f.axis == 1 ? oy : oz);
    o[f.e] = mac_sample_comp(mac, q, f.axis);
}

struct Face3 {
    const float* p[3];
    // select with constant indices only: a run-time index into a kernel
    // parameter array makes the compiler copy the parameter to local memory
    EDGE_D const float* at(int a) const { return a == 0 ? p[0] : (a == 1 ? p[1] : p[2]); }
};

// map_u / map_u_psi pullback with fused BFECC arithmetic (edge_pullback_u)
template <bool P2>
__global__ void __launch_bounds__(256) k_pullback_u(Mac mac_, Face3 pos, Face3 col, Face3 init, float scale, Face3 sub,
                                                    float* ox, float* oy, float* oz) {
    const Mac mac = with_pow2<P2>(mac_);
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_faces(mac.nx, mac.ny, mac.nz)) return;
    FaceIdx f = face_decompose(t, mac.nx, mac.ny, mac.nz);
    const float* P = pos.at(f.axis) + 3 * f.e;
    const float* Cc = col.at(f.axis) + 3 * f.e;
    float p[3] = {__ldg(P), __ldg(P + 1), __ldg(P + 2)};
    float v[3];
    mac_sample<false>(mac, p, v, nullptr);
    float out = __ldg(Cc) * v[0] + __ldg(Cc + 1) * v[1] + __ldg(Cc + 2) * v[2];
    if (init.at(f.axis)) out = scale * (out - __ldg(init.at(f.axis) + f.e));
    if (sub.at(f.axis)) out = __ldg(sub.at(f.axis) + f.e) - out;
    float* o = f.axis == 0 ? ox : (f.axis == 1 ? oy : oz);
    o[f.e] = out;
}

// map_u_psi straight from the cell map (run_edge.py:377-417, run_ed4.py:219-260)
template <int V>
__global__ void __launch_bounds__(128) k_map_u_psi(Mac mac, MapF m, float* ox, float* oy, float* oz) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_faces(m.nx, m.ny, m.nz)) return;
    FaceIdx f = face_decompose(t, m.nx, m.ny, m.nz);
    float X[3], P[3], G[3][3], v[3];
    face_pos(f.axis, f.i, f.j, f.k, m.dx, X);
    hermite3<V, true>(m, X, P, G);
    mac_sample<false>(mac, P, v, nullptr);
    float out = sel3(G[0], f.axis) * v[0] + sel3(G[1], f.axis) * v[1] + sel3(G[2], f.axis) * v[2];
    float* o = f.axis == 0 ? ox : (f.axis == 1 ? oy : oz);
    o[f.e] = out;
}

// cell centre of the map = mean of the six face positions (run_edge.py:424-426, 460-461)
EDGE_D void centre_from_faces(const Face3& pos, int nx, int ny, int nz, int i, int j, int k, float pc[3]) {
    const float* a0 = pos.p[0] + 3 * idx3(i, j, k, ny, nz);
    const float* a1 = pos.p[0] + 3 * idx3(i + 1, j, k, ny, nz);
    const float* b0 = pos.p[1] + 3 * idx3(i, j, k, ny + 1, nz);
    const float* b1 = pos.p[1] + 3 * idx3(i, j + 1, k, ny + 1, nz);
    const float* c0 = pos.p[2] + 3 * idx3(i, j, k, ny, nz + 1);
    const float* c1 = pos.p[2] + 3 * idx3(i, j, k + 1, ny, nz + 1);
    for (int c = 0; c < 3; c++)
        pc[c] = (1.0f / 6.0f) *
                (__ldg(a0 + c) + __ldg(a1 + c) + __ldg(b0 + c) + __ldg(b1 + c) + __ldg(c0 + c) + __ldg(c1 + c));
}

template <bool P2>
__global__ void __launch_bounds__(256) k_pullback_dye(Dye dye_, const float* __restrict__ smoke0, Face3 pos,
                                                      const float* __restrict__ init, float scale,
                                                      const float* sub, const float* __restrict__ clampsrc,
                                                      int inplace_clamp, float* out) {
    const Dye dye = with_pow2<P2>(dye_);
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    int n = dye.nx * dye.ny * dye.nz;
    if (e >= n) return;
    int k = e % dye.nz, j = (e / dye.nz) % dye.ny, i = e / (dye.ny * dye.nz);
    float pc[3];
    centre_from_faces(pos, dye.nx, dye.ny, dye.nz, i, j, k, pc);
    Lin8 L = lin_setup(dye, pc);
    float4 v;
    if (inplace_clamp) {
        v = reinterpret_cast<const float4*>(out)[e];
    } else {
        v = dye_interp(smoke0, dye, L);
        if (init) {
            float4 a = ld4(init, e);
            v = make_float4(scale * (v.x - a.x), scale * (v.y - a.y), scale * (v.z - a.z), scale * (v.w - a.w));
        }
        if (sub) {
            float4 a = reinterpret_cast<const float4*>(sub)[e];
            v = make_float4(a.x - v.x, a.y - v.y, a.z - v.z, a.w - v.w);
        }
    }
    if (clampsrc) {
        float4 mn, mx;
        dye_minmax(clampsrc, dye, L, mn, mx);
        v = clamp4(v, mn, mx);
    }
    reinterpret_cast<float4*>(out)[e] = v;
}

// map_smoke_psi (MODE 0) / clamp_smoke_psi (MODE 1) from the cell map
template <int V, int MODE>
__global__ void __launch_bounds__(128) k_smoke_psi(Dye dye, MapF m, const float* __restrict__ smoke0, float* out) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    int n = m.nx * m.ny * m.nz;
    if (e >= n) return;
    int k = e % m.nz, j = (e / m.nz) % m.ny, i = e / (m.ny * m.nz);
    float s[3] = {0.f, 0.f, 0.f};
#pragma unroll 1
    for (int q = 0; q < 6; q++) {
        int a = q >> 1, side = q & 1;
        float X[3], v[3];
        face_pos(a, i + (a == 0 ? side : 0), j + (a == 1 ? side : 0), k + (a == 2 ? side : 0), m.dx, X);
        hermite3<V, false>(m, X, v, nullptr);
        for (int c = 0; c < 3; c++) s[c] += v[c];
    }
    float pc[3] = {(1.0f / 6.0f) * s[0], (1.0f / 6.0f) * s[1], (1.0f / 6.0f) * s[2]};
    Lin8 L = lin_setup(dye, pc);
    float4* o = reinterpret_cast<float4*>(out);
    if (MODE == 0) {
        o[e] = dye_interp(smoke0, dye, L);
    } else {
        float4 mn, mx;
        dye_minmax(smoke0, dye, L, mn, mx);
        o[e] = clamp4(o[e], mn, mx);
    }
}

// clamp_u (run_edge.py:509-519) over the three face grids
__global__ void k_clamp_u(int nx, int ny, int nz, Face3 u, Face3 u1, float* ox, float* oy, float* oz) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_faces(nx, ny, nz)) return;
    FaceIdx f = face_decompose(t, nx, ny, nz);
    int n0 = nx + (f.axis == 0), n1 = ny + (f.axis == 1), n2 = nz + (f.axis == 2);
    const float* a = u1.at(f.axis);
    int im = max(f.i - 1, 0), ip = min(f.i + 1, n0 - 1);
    int jm = max(f.j - 1, 0), jp = min(f.j + 1, n1 - 1);
    int km = max(f.k - 1, 0), kp = min(f.k + 1, n2 - 1);
    float l = __ldg(a + idx3(im, f.j, f.k, n1, n2)), r = __ldg(a + idx3(ip, f.j, f.k, n1, n2));
    float b = __ldg(a + idx3(f.i, jm, f.k, n1, n2)), tt = __ldg(a + idx3(f.i, jp, f.k, n1, n2));
    float aa = __ldg(a + idx3(f.i, f.j, km, n1, n2)), cc = __ldg(a + idx3(f.i, f.j, kp, n1, n2));
    float mx = fmaxf(fmaxf(fmaxf(fmaxf(fmaxf(l, r), b), tt), aa), cc);
    float mn = fminf(fminf(fminf(fminf(fminf(l, r), b), tt), aa), cc);
    float* o = f.axis == 0 ? ox : (f.axis == 1 ? oy : oz);
    o[f.e] = fminf(fmaxf(__ldg(u.at(f.axis) + f.e), mn), mx);
}

__global__ void k_set_float(float* p, float v) { *p = v; }

// calc_max_speed (run_edge.py:296-303): block max + atomicMax on the float's
// bits (speeds are non-negative, so integer order is float order).
__global__ void k_max_speed(int nx, int ny, int nz, const float* __restrict__ ux, const float* __restrict__ uy,
                            const float* __restrict__ uz, float* out) {
    int n = nx * ny * nz;
    float best = 0.0f;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        int k = e % nz, j = (e / nz) % ny, i = e / (ny * nz);
        float u = 0.5f * (__ldg(ux + idx3(i, j, k, ny, nz)) + __ldg(ux + idx3(i + 1, j, k, ny, nz)));
        float v = 0.5f * (__ldg(uy + idx3(i, j, k, ny + 1, nz)) + __ldg(uy + idx3(i, j + 1, k, ny + 1, nz)));
        float w = 0.5f * (__ldg(uz + idx3(i, j, k, ny, nz + 1)) + __ldg(uz + idx3(i, j, k + 1, ny, nz + 1)));
        best = fmaxf(best, sqrtf(u * u + v * v + w * w));
    }
    for (int o = 16; o > 0; o >>= 1) best = fmaxf(best, __shfl_xor_sync(0xffffffffu, best, o));
    __shared__ float sm[32];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sm[wid] = best;
    __syncthreads();
    if (wid == 0) {
        best = lane < (int)(blockDim.x >> 5) ? sm[lane] : 0.0f;
        for (int o = 16; o > 0; o >>= 1) best = fmaxf(best, __shfl_xor_sync(0xffffffffu, best, o));
        if (lane == 0) atomicMax(reinterpret_cast<int*>(out), __float_as_int(best));
    }
}

// run_edge.py:595-614 on the device (doubles as the driver's Python floats)
__global__ void k_compute_dt(const float* ms, double cfl_dx, double visualize_dt, double* st, float* dt_out,
                             float* half_out) {
    double cur = cfl_dx / (double)(*ms);
    double sub_t = st[0];
    double frame = st[1];
    double output = 0.0;
    if (sub_t + cur >= visualize_dt) {
        cur = visualize_dt - sub_t;
        sub_t = 0.0;
        frame += 1.0;
        output = 1.0;
    } else if (sub_t + cur * 2.0 >= visualize_dt) {
        cur = (visualize_dt - sub_t) / 2.0;
        sub_t += cur;
    } else {
        sub_t += cur;
    }
    st[0] = sub_t;
    st[1] = frame;
    st[2] = output;
    st[3] = cur;
    *dt_out = (float)cur;
    *half_out = (float)(0.5 * cur);
}

__global__ void k_axpy(long long n, const float* __restrict__ f1, const float* __restrict__ f2, float a,
                       float* dest) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        dest[e] = f2 ? f1[e] + a * f2[e] : a * f1[e];
}

// ---------------------------------------------------------------------------
// initial conditions (init_conditions.py:11-36, taichi_utils.py:103-116)
// ---------------------------------------------------------------------------
struct Ring {
    float w, rad, delta, c[3], ex[3], ey[3], color[3];
    int ns;
};
__global__ void k_vortex_ring(int nx, int ny, int nz, float dx, Ring R, float* u, float* smoke) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nx * ny * nz) return;
    int k = e % nz, j = (e / nz) % ny, i = e / (ny * nz);
    const float PI = 3.14159265358979323846f;
    float X[3];
    cell_pos(i, j, k, dx, X);
    float curve = (2.0f * PI * R.rad) / (float)R.ns;
    float acc[3] = {u[3 * e], u[3 * e + 1], u[3 * e + 2]};
    float sm = smoke[4 * e + 3];
    for (int l = 0; l < R.ns; l++) {
        float th = (float)l / (float)R.ns * 2.0f * PI;
        float ct = cosf(th), st = sinf(th), d[3], wv[3];
        for (int c = 0; c < 3; c++) d[c] = X[c] - (R.rad * (ct * R.ex[c] + st * R.ey[c]) + R.c[c]);
        float r = sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        for (int c = 0; c < 3; c++) wv[c] = R.w * (-st * R.ex[c] + ct * R.ey[c]);
        float q = r / R.delta;
        float ex = expf(-(q * q * q));
        float fac = curve * (-1.0f / (4.0f * PI * (r * r * r)) * (1.0f - ex));
        acc[0] += fac * (d[1] * wv[2] - d[2] * wv[1]);
        acc[1] += fac * (d[2] * wv[0] - d[0] * wv[2]);
        acc[2] += fac * (d[0] * wv[1] - d[1] * wv[0]);
        sm += curve * ex;
    }
    for (int c = 0; c < 3; c++) u[3 * e + c] = acc[c];
    if (sm > 0.002f) {
        smoke[4 * e + 0] = R.color[0];
        smoke[4 * e + 1] = R.color[1];
        smoke[4 * e + 2] = R.color[2];
        smoke[4 * e + 3] = 1.0f;
    } else {
        smoke[4 * e + 0] = smoke[4 * e + 1] = smoke[4 * e + 2] = smoke[4 * e + 3] = 0.0f;
    }
}

__global__ void k_split_central(int nx, int ny, int nz, const float* __restrict__ vc, float* ux, float* uy,
                                float* uz) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_faces(nx, ny, nz)) return;
    FaceIdx f = face_decompose(t, nx, ny, nz);
    int hi[3] = {min(f.i, nx - 1), min(f.j, ny - 1), min(f.k, nz - 1)};
    int lo[3] = {f.axis == 0 ? max(f.i - 1, 0) : hi[0], f.axis == 1 ? max(f.j - 1, 0) : hi[1],
                 f.axis == 2 ? max(f.k - 1, 0) : hi[2]};
    float r = vc[3 * idx3(hi[0], hi[1], hi[2], ny, nz) + f.axis];
    float l = vc[3 * idx3(lo[0], lo[1], lo[2], ny, nz) + f.axis];
    float* o = f.axis == 0 ? ux : (f.axis == 1 ? uy : uz);
    o[f.e] = 0.5f * (r + l);
}

// get_central_vector (taichi_utils.py:95-100): the face average per cell
__global__ void k_get_central(int nx, int ny, int nz, const float* __restrict__ ux, const float* __restrict__ uy,
                              const float* __restrict__ uz, float* __restrict__ vc) {
    long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)nx * ny * nz) return;
    int k = (int)(e % nz), j = (int)((e / nz) % ny), i = (int)(e / ((long long)ny * nz));
    float x = 0.5f * (ux[idx3(i + 1, j, k, ny, nz)] + ux[idx3(i, j, k, ny, nz)]);
    float y = 0.5f * (uy[idx3(i, j + 1, k, ny + 1, nz)] + uy[idx3(i, j, k, ny + 1, nz)]);
    float z = 0.5f * (uz[idx3(i, j, k + 1, ny, nz + 1)] + uz[idx3(i, j, k, ny, nz + 1)]);
    vc[3 * e] = x;
    vc[3 * e + 1] = y;
    vc[3 * e + 2] = z;
}

// curl (taichi_utils.py:69-92): central differences of a cell vec3 field with
// the neighbour index clamped to the grid (sample, taichi_utils.py:61-66);
// products by 1/(2dx) rounded before the difference, as the reference's
// separate statements round them
__global__ void k_curl(int nx, int ny, int nz, float dx, const float* __restrict__ vf, float* __restrict__ cf) {
    long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)nx * ny * nz) return;
    int k = (int)(e % nz), j = (int)((e / nz) % ny), i = (int)(e / ((long long)ny * nz));
    const float inv = 1.0f / (2.0f * dx);
    auto at = [&](int a, int b, int c) {
        a = max(0, min(a, nx - 1));
        b = max(0, min(b, ny - 1));
        c = max(0, min(c, nz - 1));
        return vf + 3 * (long long)idx3(a, b, c, ny, nz);
    };
    const float *vr = at(i + 1, j, k), *vl = at(i - 1, j, k), *vt = at(i, j + 1, k), *vb = at(i, j - 1, k),
                *vc = at(i, j, k + 1), *va = at(i, j, k - 1);
    float dvx_dz = __fmul_rn(inv, __fsub_rn(vc[0], va[0]));
    float dvx_dy = __fmul_rn(inv, __fsub_rn(vt[0], vb[0]));
    float dvy_dx = __fmul_rn(inv, __fsub_rn(vr[1], vl[1]));
    float dvy_dz = __fmul_rn(inv, __fsub_rn(vc[1], va[1]));
    float dvz_dx = __fmul_rn(inv, __fsub_rn(vr[2], vl[2]));
    float dvz_dy = __fmul_rn(inv, __fsub_rn(vt[2], vb[2]));
    cf[3 * e] = __fsub_rn(dvz_dy, dvy_dz);
    cf[3 * e + 1] = __fsub_rn(dvx_dz, dvz_dx);
    cf[3 * e + 2] = __fsub_rn(dvy_dx, dvx_dy);
}

// emit_smoke_delta (init_conditions.py:177-232): cells whose centre lies
// within `radius` of an emitter take its colour; later emitters win, as the
// reference's sequence of ifs does.
struct Emitters {
    float c[16][3];
    float col[16][4];
    int k;
    float radius;
};
__global__ void k_emit_spheres(int nx, int ny, int nz, float dx, Emitters E, float4* smoke) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nx * ny * nz) return;
    int k = e % nz, j = (e / nz) % ny, i = e / (ny * nz);
    float X[3];
    cell_pos(i, j, k, dx, X);
    for (int q = 0; q < E.k; q++) {
        float d0 = X[0] - E.c[q][0], d1 = X[1] - E.c[q][1], d2 = X[2] - E.c[q][2];
        if (sqrtf(d0 * d0 + d1 * d1 + d2 * d2) < E.radius)
            smoke[e] = make_float4(E.col[q][0], E.col[q][1], E.col[q][2], E.col[q][3]);
    }
}

// clamp_smoke_density (init_conditions.py:234-243)
__global__ void k_clamp_max(long long n, float hi, float* x) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        if (x[e] > hi) x[e] = hi;
}

inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int edge_version(void) { return 10000; }

const char* edge_error_string(int code) {
    switch (code) {
        case EDGE_OK: return "ok";
        case EDGE_EINVAL: return "invalid argument (sizes, null pointer or option)";
        case EDGE_EALIGN: return "misaligned pointer (vec4 fields need 16-byte alignment)";
        case EDGE_ENOCONV: return "solver reached max_iters without converging";
        case EDGE_ENAN: return "non-finite residual";
        case EDGE_ESTALL: return "residual stalled";
        case EDGE_ESTATE: return "invalid call order or handle state";
        default: return code > 0 ? cudaGetErrorString((cudaError_t)code) : "unknown error";
    }
}

int edge_points_mac(int nx, int ny, int nz, float dx, const float* ux, const float* uy, const float* uz,
                    const float* pts, int n, float* v, float* vg, float* g, void* stream) {
    if (!dims_ok(nx, ny, nz) || n < 0 || !ux || !uy || !uz || (n && (!pts || !v || !vg || !g))) return EDGE_EINVAL;
    if (n == 0) return EDGE_OK;
    k_points_mac<<<grid_for(n), kBlock, 0, S(stream)>>>(make_mac(ux, uy, uz, nx, ny, nz, dx), pts, n, v, vg, g);
    return launch_status();
}

int edge_points_dye(int nx, int ny, int nz, float dx, const float* smoke, const float* pts, int n, float* lin,
                    float* mn, float* mx, void* stream) {
    if (!dims_ok(nx, ny, nz) || n < 0 || !smoke || (n && (!pts || !lin || !mn || !mx))) return EDGE_EINVAL;
    if (!al16(smoke) || !al16(lin) || !al16(mn) || !al16(mx)) return EDGE_EALIGN;
    if (n == 0) return EDGE_OK;
    k_points_dye<<<grid_for(n), kBlock, 0, S(stream)>>>(make_dye(nx, ny, nz, dx), smoke, pts, n, (float4*)lin,
                                                        (float4*)mn, (float4*)mx);
    return launch_status();
}

int edge_points_hermite(int variant, int nx, int ny, int nz, float dx, const float* psi, const float* Tx,
                        const float* Ty, const float* Tz, const float* dTx, const float* dTy, const float* dTz,
                        const float* d2Tx, const float* d2Ty, const float* d2Tz, const float* pts, int n,
                        float* val, float* gval, float* grad, void* stream) {
    if (!dims_ok(nx, ny, nz) || n < 0 || !psi || !Tx || !Ty || !Tz) return EDGE_EINVAL;
    if (variant != HV_FD && (!dTx || !dTy || !dTz)) return EDGE_EINVAL;
    if (variant == HV_FULL && (!d2Tx || !d2Ty || !d2Tz)) return EDGE_EINVAL;
    if (n == 0) return EDGE_OK;
    const float* T[3] = {Tx, Ty, Tz};
    const float* dT[3] = {dTx, dTy, dTz};
    const float* d2T[3] = {d2Tx, d2Ty, d2Tz};
    MapF m = make_map(psi, T, dT, d2T, nx, ny, nz, dx);
    if (variant == HV_FD) k_points_hermite<HV_FD><<<grid_for(n), kBlock, 0, S(stream)>>>(m, pts, n, val, gval, grad);
    else if (variant == HV_GARM) k_points_hermite<HV_GARM><<<grid_for(n), kBlock, 0, S(stream)>>>(m, pts, n, val, gval, grad);
    else if (variant == HV_FULL) k_points_hermite<HV_FULL><<<grid_for(n), kBlock, 0, S(stream)>>>(m, pts, n, val, gval, grad);
    else return EDGE_EINVAL;
    return launch_status();
}

int edge_reset_cells(int nx, int ny, int nz, float dx, float* psi, float* Tx, float* Ty, float* Tz, float* dTx,
                     float* dTy, float* dTz, float* d2Tx, float* d2Ty, float* d2Tz, void* stream) {
    if (!dims_ok(nx, ny, nz) || !psi || !Tx || !Ty || !Tz) return EDGE_EINVAL;
    int n = nx * ny * nz;
    k_reset_cells<<<grid_for(n), kBlock, 0, S(stream)>>>(nx, ny, nz, dx, psi, Tx, Ty, Tz, dTx, dTy, dTz, d2Tx, d2Ty,
                                                         d2Tz);
    return launch_status();
}

int edge_reset_faces(int nx, int ny, int nz, float dx, float* phix, float* phiy, float* phiz, float* Fx, float* Fy,
                     float* Fz, void* stream) {
    if (!dims_ok(nx, ny, nz) || !phix || !phiy || !phiz || !Fx || !Fy || !Fz) return EDGE_EINVAL;
    k_reset_faces<<<grid_for(n_faces(nx, ny, nz)), kBlock, 0, S(stream)>>>(nx, ny, nz, dx, phix, phiy, phiz, Fx,
                                                                           Fy, Fz);
    return launch_status();
}

int edge_march_edge(int nx, int ny, int nz, float dx, float dt, float epsilon, const float* ux, const float* uy,
                    const float* uz, const float* psi, const float* Tx, const float* Ty, const float* Tz,
                    const float* dTx, const float* dTy, const float* dTz, float* opsi, float* oTx, float* oTy,
                    float* oTz, float* odTx, float* odTy, float* odTz, int identity, void* stream) {
    if (!dims_ok(nx, ny, nz) || !ux || !uy || !uz || !opsi || !oTx || !oTy || !oTz || !odTx || !odTy || !odTz)
        return EDGE_EINVAL;
    if (!identity && (!psi || !Tx || !Ty || !Tz || !dTx || !dTy || !dTz)) return EDGE_EINVAL;
    if (!identity && (opsi == psi || oTx == Tx || odTx == dTx)) return EDGE_EINVAL;
    const float* T[3] = {Tx, Ty, Tz};
    const float* dT[3] = {dTx, dTy, dTz};
    MapF m = make_map(psi, T, dT, nullptr, nx, ny, nz, dx);
    Mac mac = make_mac(ux, uy, uz, nx, ny, nz, dx);
    int n = nx * ny * nz;
    if (identity)
        k_march_edge<true><<<grid_for(n, 128), 128, 0, S(stream)>>>(mac, m, dt, epsilon, opsi, oTx, oTy, oTz, odTx,
                                                                    odTy, odTz);
    else
        k_march_edge<false><<<grid_for(n, 128), 128, 0, S(stream)>>>(mac, m, dt, epsilon, opsi, oTx, oTy, oTz, odTx,
                                                                     odTy, odTz);
    return launch_status();
}

int edge_march_ed4(int nx, int ny, int nz, float dx, float dt, float epsilon, const float* ux, const float* uy,
                   const float* uz, const float* psi, const float* Tx, const float* Ty, const float* Tz, float* opsi,
                   float* oTx, float* oTy, float* oTz, void* stream) {
    if (!dims_ok(nx, ny, nz) || !ux || !uy || !uz || !psi || !Tx || !Ty || !Tz || !opsi || !oTx || !oTy || !oTz)
        return EDGE_EINVAL;
    if (opsi == psi || oTx == Tx || oTy == Ty || oTz == Tz) return EDGE_EINVAL;
    const float* T[3] = {Tx, Ty, Tz};
    MapF m = make_map(psi, T, nullptr, nullptr, nx, ny, nz, dx);
    int n = nx * ny * nz;
    k_march_ed4<<<grid_for(n, 128), 128, 0, S(stream)>>>(make_mac(ux, uy, uz, nx, ny, nz, dx), m, dt, epsilon, opsi,
                                                        oTx, oTy, oTz);
    return launch_status();
}

int edge_march_ed8(int nx, int ny, int nz, float dx, float dt, float epsilon, const float* ux, const float* uy,
                   const float* uz, const float* psi, const float* Tx, const float* Ty, const float* Tz,
                   const float* dTx, const float* dTy, const float* dTz, const float* d2Tx, const float* d2Ty,
                   const float* d2Tz, float* opsi, float* oTx, float* oTy, float* oTz, float* odTx, float* odTy,
                   float* odTz, float* od2Tx, float* od2Ty, float* od2Tz, void* stream) {
    if (!dims_ok(nx, ny, nz) || !ux || !uy || !uz || !psi || !Tx || !Ty || !Tz || !dTx || !dTy || !dTz || !d2Tx ||
        !d2Ty || !d2Tz || !opsi || !oTx || !oTy || !oTz || !odTx || !odTy || !odTz || !od2Tx || !od2Ty || !od2Tz)
        return EDGE_EINVAL;
    if (opsi == psi || oTx == Tx || odTx == dTx || od2Tx == d2Tx) return EDGE_EINVAL;
    const float* T[3] = {Tx, Ty, Tz};
    const float* dT[3] = {dTx, dTy, dTz};
    const float* d2T[3] = {d2Tx, d2Ty, d2Tz};
    MapF m = make_map(psi, T, dT, d2T, nx, ny, nz, dx);
    int n = nx * ny * nz;
    k_march_ed8<<<grid_for(n, 128), 128, 0, S(stream)>>>(make_mac(ux, uy, uz, nx, ny, nz, dx), m, dt, epsilon, opsi,
                                                        oTx, oTy, oTz, odTx, odTy, odTz, od2Tx, od2Ty, od2Tz);
    return launch_status();
}

int edge_calc_fd_3_from_grad(int nx, int ny, int nz, float dx, const float* Tx, const float* Ty, const float* Tz,
                             float* dTx, float* dTy, float* dTz, float* d2Tx, float* d2Ty, float* d2Tz, void* stream) {
    if (!dims_ok(nx, ny, nz) || !Tx || !Ty || !Tz || !dTx || !dTy || !dTz || !d2Tx || !d2Ty || !d2Tz)
        return EDGE_EINVAL;
    if (dTx == Tx || dTy == Ty || dTz == Tz) return EDGE_EINVAL;
    long long n3 = 3LL * nx * ny * nz;
    k_fd3_dT<<<grid_for(n3), kBlock, 0, S(stream)>>>(nx, ny, nz, dx, Tx, Ty, Tz, dTx, dTy, dTz);
    k_fd3_d2T<<<grid_for(n3), kBlock, 0, S(stream)>>>(nx, ny, nz, dx, dTx, dTy, dTz, d2Tx, d2Ty, d2Tz);
    return launch_status();
}

int edge_march_ge(int nx, int ny, int nz, float dx, float dt, const float* ux, const float* uy, const float* uz,
                  const float* psi, const float* Tx, const float* Ty, const float* Tz, const float* dTx,
                  const float* dTy, const float* dTz, const float* d2Tx, const float* d2Ty, const float* d2Tz,
                  float* opsi, float* oTx, float* oTy, float* oTz, float* odTx, float* odTy, float* odTz,
                  float* od2Tx, float* od2Ty, float* od2Tz, void* stream) {
    if (!dims_ok(nx, ny, nz) || !ux || !uy || !uz || !psi || !Tx || !Ty || !Tz || !dTx || !dTy || !dTz || !d2Tx ||
        !d2Ty || !d2Tz || !opsi || !oTx || !oTy || !oTz || !odTx || !odTy || !odTz || !od2Tx || !od2Ty || !od2Tz)
        return EDGE_EINVAL;
    if (opsi == psi || oTx == Tx || odTx == dTx || od2Tx == d2Tx) return EDGE_EINVAL;
    const float* T[3] = {Tx, Ty, Tz};
    const float* dT[3] = {dTx, dTy, dTz};
    const float* d2T[3] = {d2Tx, d2Ty, d2Tz};
    MapF m = make_map(psi, T, dT, d2T, nx, ny, nz, dx);
    int n = nx * ny * nz;
    k_march_ge<<<grid_for(n, 128), 128, 0, S(stream)>>>(make_mac(ux, uy, uz, nx, ny, nz, dx), m, dt, opsi, oTx, oTy,
                                                       oTz);
    int rc = launch_status();
    if (rc) return rc;
    return edge_calc_fd_3_from_grad(nx, ny, nz, dx, oTx, oTy, oTz, odTx, odTy, odTz, od2Tx, od2Ty, od2Tz, stream);
}

int edge_march_ge_packed(int nx, int ny, int nz, float dx, float dt, const float* ux, const float* uy,
                         const float* uz, const float* in_packed, float* out_packed, void* stream) {
    if (!dims_ok(nx, ny, nz) || !ux || !uy || !uz || !in_packed || !out_packed) return EDGE_EINVAL;
    if (in_packed == out_packed) return EDGE_EINVAL;
    if (!al16(in_packed) || !al16(out_packed)) return EDGE_EALIGN;
    MapP m = make_mapp(in_packed, nx, ny, nz, dx);
    int n = nx * ny * nz;
    float4* o = (float4*)out_packed;
    const Mac mac = make_mac(ux, uy, uz, nx, ny, nz, dx);
    if (mac.pow2) k_march_ge_p<false, true><<<grid_for(n, 128), 128, 0, S(stream)>>>(mac, m, dt, o);
    else k_march_ge_p<false, false><<<grid_for(n, 128), 128, 0, S(stream)>>>(mac, m, dt, o);
    k_fd3_dT_p<<<grid_for(n), kBlock, 0, S(stream)>>>(nx, ny, nz, dx, o);
    k_fd3_d2T_p<<<grid_for(n), kBlock, 0, S(stream)>>>(nx, ny, nz, dx, o);
    return launch_status();
}

static int planes_of(int variant) {
    return variant == HV_FD ? kPlanesED4 : (variant == HV_GARM ? kPlanesEDGE : (variant == HV_FULL ? kPlanesED8 : -1));
}

// fill the derived coefficient planes of a packed ED4 / EDGE map
static void derive_planes(int variant, int nx, int ny, int nz, float* packed, cudaStream_t st) {
    MapP m = make_mapp(packed, nx, ny, nz, 1.0f);
    int n = nx * ny * nz;
    if (variant == HV_FD) k_coef_p<HV_FD><<<grid_for(n), kBlock, 0, st>>>(m, (float4*)packed);
    else if (variant == HV_GARM) k_coef_p<HV_GARM><<<grid_for(n), kBlock, 0, st>>>(m, (float4*)packed);
}

int edge_map_pack(int variant, int nx, int ny, int nz, const float* psi, const float* Tx, const float* Ty,
                  const float* Tz, const float* dTx, const float* dTy, const float* dTz, const float* d2Tx,
                  const float* d2Ty, const float* d2Tz, float* packed, void* stream) {
    int pl = planes_of(variant);
    if (!dims_ok(nx, ny, nz) || pl < 0 || !psi || !Tx || !Ty || !Tz || !packed) return EDGE_EINVAL;
    if (pl >= 7 && (!dTx || !dTy || !dTz)) return EDGE_EINVAL;
    if (pl >= 8 && (!d2Tx || !d2Ty || !d2Tz)) return EDGE_EINVAL;
    if (!al16(packed)) return EDGE_EALIGN;
    int n = nx * ny * nz;
    k_map_pack<<<grid_for(n), kBlock, 0, S(stream)>>>(n, pl, psi, Tx, Ty, Tz, dTx, dTy, dTz, d2Tx, d2Ty, d2Tz,
                                                      (float4*)packed);
    derive_planes(variant, nx, ny, nz, packed, S(stream));
    return launch_status();
}

int edge_packed_planes(int variant) { return planes_of(variant) < 0 ? EDGE_EINVAL : kPlanesStored; }

int edge_map_unpack(int variant, int nx, int ny, int nz, const float* packed, float* psi, float* Tx, float* Ty,
                    float* Tz, float* dTx, float* dTy, float* dTz, float* d2Tx, float* d2Ty, float* d2Tz,
                    void* stream) {
    int pl = planes_of(variant);
    if (!dims_ok(nx, ny, nz) || pl < 0 || !psi || !Tx || !Ty || !Tz || !packed) return EDGE_EINVAL;
    if (pl >= 7 && (!dTx || !dTy || !dTz)) return EDGE_EINVAL;
    if (pl >= 8 && (!d2Tx || !d2Ty || !d2Tz)) return EDGE_EINVAL;
    if (!al16(packed)) return EDGE_EALIGN;
    int n = nx * ny * nz;
    k_map_unpack<<<grid_for(n), kBlock, 0, S(stream)>>>(n, pl, (const float4*)packed, psi, Tx, Ty, Tz, dTx, dTy,
                                                        dTz, d2Tx, d2Ty, d2Tz);
    return launch_status();
}

int edge_march_packed(int variant, int nx, int ny, int nz, float dx, float dt, float epsilon, const float* ux,
                      const float* uy, const float* uz, const float* in_packed, float* out_packed, int flags,
                      void* stream) {
    int pl = planes_of(variant);
    if (flags & ~(EDGE_MARCH_IDENTITY | EDGE_MARCH_F64_COMPOSE)) return EDGE_EINVAL;
    const int identity = flags & EDGE_MARCH_IDENTITY, f64 = (flags & EDGE_MARCH_F64_COMPOSE) != 0;
    if (!dims_ok(nx, ny, nz) || pl < 0 || !ux || !uy || !uz || !out_packed) return EDGE_EINVAL;
    if (!identity && !in_packed) return EDGE_EINVAL;
    if (identity && variant != HV_GARM) return EDGE_EINVAL;
    if (in_packed == out_packed) return EDGE_EINVAL;
    if (!al16(in_packed) || !al16(out_packed)) return EDGE_EALIGN;
    MapP m = make_mapp(in_packed, nx, ny, nz, dx);
    Mac mac = make_mac(ux, uy, uz, nx, ny, nz, dx);
    int n = nx * ny * nz;
    float4* o = (float4*)out_packed;
    if (variant == HV_GARM) {
        const int g = grid_for(n, 128);
        if (mac.pow2) {
            if (identity) k_march_edge_p<true, false, true><<<g, 128, 0, S(stream)>>>(mac, m, dt, epsilon, o);
            else if (f64) k_march_edge_p<false, true, true><<<g, 128, 0, S(stream)>>>(mac, m, dt, epsilon, o);
            else k_march_edge_p<false, false, true><<<g, 128, 0, S(stream)>>>(mac, m, dt, epsilon, o);
        } else {
            if (identity) k_march_edge_p<true, false, false><<<g, 128, 0, S(stream)>>>(mac, m, dt, epsilon, o);
            else if (f64) k_march_edge_p<false, true, false><<<g, 128, 0, S(stream)>>>(mac, m, dt, epsilon, o);
            else k_march_edge_p<false, false, false><<<g, 128, 0, S(stream)>>>(mac, m, dt, epsilon, o);
        }
    } else if (variant == HV_FD) {
        if (mac.pow2) k_march_ed4_p<true><<<grid_for(n, 128), 128, 0, S(stream)>>>(mac, m, dt, epsilon, o);
        else k_march_ed4_p<false><<<grid_for(n, 128), 128, 0, S(stream)>>>(mac, m, dt, epsilon, o);
    } else {
        if (mac.pow2) k_march_ed8_p<true><<<grid_for(n, 128), 128, 0, S(stream)>>>(mac, m, dt, epsilon, o);
        else k_march_ed8_p<false><<<grid_for(n, 128), 128, 0, S(stream)>>>(mac, m, dt, epsilon, o);
    }
    derive_planes(variant, nx, ny, nz, out_packed, S(stream));
    return launch_status();
}

int edge_face_map_packed(int variant, int nx, int ny, int nz, float dx, const float* packed, float* fpsix,
                         float* fpsiy, float* fpsiz, float* fcolx, float* fcoly, float* fcolz, void* stream) {
    if (!dims_ok(nx, ny, nz) || planes_of(variant) < 0 || !packed || !fpsix || !fpsiy || !fpsiz || !fcolx ||
        !fcoly || !fcolz)
        return EDGE_EINVAL;
    if (!al16(packed)) return EDGE_EALIGN;
    MapP m = make_mapp(packed, nx, ny, nz, dx);
    const int gx = grid_for((long long)(nx + 1) * ny * nz, 128), gy = grid_for((long long)nx * (ny + 1) * nz, 128),
              gz = grid_for((long long)nx * ny * (nz + 1), 128);
    cudaStream_t st = S(stream);
    if (variant == HV_FD) {
        if (m.pow2) {
            k_face_map_p<HV_FD_P, 0, true><<<gx, 128, 0, st>>>(m, fpsix, fcolx);
            k_face_map_p<HV_FD_P, 1, true><<<gy, 128, 0, st>>>(m, fpsiy, fcoly);
            k_face_map_p<HV_FD_P, 2, true><<<gz, 128, 0, st>>>(m, fpsiz, fcolz);
        } else {
            k_face_map_p<HV_FD_P, 0, false><<<gx, 128, 0, st>>>(m, fpsix, fcolx);
            k_face_map_p<HV_FD_P, 1, false><<<gy, 128, 0, st>>>(m, fpsiy, fcoly);
            k_face_map_p<HV_FD_P, 2, false><<<gz, 128, 0, st>>>(m, fpsiz, fcolz);
        }
    } else if (variant == HV_GARM) {
        if (m.pow2) {
            k_face_map_p<HV_GARM_P, 0, true><<<gx, 128, 0, st>>>(m, fpsix, fcolx);
            k_face_map_p<HV_GARM_P, 1, true><<<gy, 128, 0, st>>>(m, fpsiy, fcoly);
            k_face_map_p<HV_GARM_P, 2, true><<<gz, 128, 0, st>>>(m, fpsiz, fcolz);
        } else {
            k_face_map_p<HV_GARM_P, 0, false><<<gx, 128, 0, st>>>(m, fpsix, fcolx);
            k_face_map_p<HV_GARM_P, 1, false><<<gy, 128, 0, st>>>(m, fpsiy, fcoly);
            k_face_map_p<HV_GARM_P, 2, false><<<gz, 128, 0, st>>>(m, fpsiz, fcolz);
        }
    } else {
        if (m.pow2) {
            k_face_map_p<HV_FULL, 0, true><<<gx, 128, 0, st>>>(m, fpsix, fcolx);
            k_face_map_p<HV_FULL, 1, true><<<gy, 128, 0, st>>>(m, fpsiy, fcoly);
            k_face_map_p<HV_FULL, 2, true><<<gz, 128, 0, st>>>(m, fpsiz, fcolz);
        } else {
            k_face_map_p<HV_FULL, 0, false><<<gx, 128, 0, st>>>(m, fpsix, fcolx);
            k_face_map_p<HV_FULL, 1, false><<<gy, 128, 0, st>>>(m, fpsiy, fcoly);
            k_face_map_p<HV_FULL, 2, false><<<gz, 128, 0, st>>>(m, fpsiz, fcolz);
        }
    }
    return launch_status();
}

int edge_face_map(int variant, int nx, int ny, int nz, float dx, const float* psi, const float* Tx, const float* Ty,
                  const float* Tz, const float* dTx, const float* dTy, const float* dTz, const float* d2Tx,
                  const float* d2Ty, const float* d2Tz, float* fpsix, float* fpsiy, float* fpsiz, float* fcolx,
                  float* fcoly, float* fcolz, void* stream) {
    if (!dims_ok(nx, ny, nz) || !psi || !Tx || !Ty || !Tz || !fpsix || !fpsiy || !fpsiz || !fcolx || !fcoly ||
        !fcolz)
        return EDGE_EINVAL;
    if (variant != HV_FD && (!dTx || !dTy || !dTz)) return EDGE_EINVAL;
    if (variant == HV_FULL && (!d2Tx || !d2Ty || !d2Tz)) return EDGE_EINVAL;
    const float* T[3] = {Tx, Ty, Tz};
    const float* dT[3] = {dTx, dTy, dTz};
    const float* d2T[3] = {d2Tx, d2Ty, d2Tz};
    MapF m = make_map(psi, T, dT, d2T, nx, ny, nz, dx);
    int g = grid_for(n_faces(nx, ny, nz), 128);
    if (variant == HV_FD) k_face_map<HV_FD><<<g, 128, 0, S(stream)>>>(m, fpsix, fpsiy, fpsiz, fcolx, fcoly, fcolz);
    else if (variant == HV_GARM) k_face_map<HV_GARM><<<g, 128, 0, S(stream)>>>(m, fpsix, fpsiy, fpsiz, fcolx, fcoly, fcolz);
    else if (variant == HV_FULL) k_face_map<HV_FULL><<<g, 128, 0, S(stream)>>>(m, fpsix, fpsiy, fpsiz, fcolx, fcoly, fcolz);
    else return EDGE_EINVAL;
    return launch_status();
}

int edge_advance_map(int nx, int ny, int nz, float dx, float dt, const float* ux, const float* uy, const float* uz,
                     float* phix, float* phiy, float* phiz, float* Fx, float* Fy, float* Fz, void* stream) {
    if (!dims_ok(nx, ny, nz) || !ux || !uy || !uz || !phix || !phiy || !phiz || !Fx || !Fy || !Fz) return EDGE_EINVAL;
    const Mac mac = make_mac(ux, uy, uz, nx, ny, nz, dx);
    const int g = grid_for(n_faces(nx, ny, nz), 128);
    if (mac.pow2) k_advance_map<true><<<g, 128, 0, S(stream)>>>(mac, dt, phix, phiy, phiz, Fx, Fy, Fz);
    else k_advance_map<false><<<g, 128, 0, S(stream)>>>(mac, dt, phix, phiy, phiz, Fx, Fy, Fz);
    return launch_status();
}

int edge_efm_backtrack(int nx, int ny, int nz, float dx, int curr_step, const float* const* ux_cache,
                       const float* const* uy_cache, const float* const* uz_cache, const float* dts, float* psix,
                       float* psiy, float* psiz, float* Tx, float* Ty, float* Tz, void* stream) {
    if (!dims_ok(nx, ny, nz) || curr_step < 0 || curr_step >= kMaxBacktrack || !ux_cache || !uy_cache ||
        !uz_cache || !dts || !psix || !psiy || !psiz || !Tx || !Ty || !Tz)
        return EDGE_EINVAL;
    VelRing ring;
    ring.steps = curr_step + 1;
    for (int s = 0; s <= curr_step; s++) {
        int src = curr_step - s;  // newest first
        if (!ux_cache[src] || !uy_cache[src] || !uz_cache[src]) return EDGE_EINVAL;
        ring.u[s][0] = ux_cache[src];
        ring.u[s][1] = uy_cache[src];
        ring.u[s][2] = uz_cache[src];
        ring.dt[s] = -dts[src];
    }
    for (int s = ring.steps; s < kMaxBacktrack; s++) {
        ring.u[s][0] = ring.u[s][1] = ring.u[s][2] = nullptr;
        ring.dt[s] = 0.0f;
    }
    const Mac mac = make_mac(ux_cache[curr_step], uy_cache[curr_step], uz_cache[curr_step], nx, ny, nz, dx);
    const int g = grid_for(n_faces(nx, ny, nz), 128);
    if (mac.pow2) k_backtrack_faces<true><<<g, 128, 0, S(stream)>>>(mac, ring, psix, psiy, psiz, Tx, Ty, Tz);
    else k_backtrack_faces<false><<<g, 128, 0, S(stream)>>>(mac, ring, psix, psiy, psiz, Tx, Ty, Tz);
    return launch_status();
}

int edge_advect_u_sl(int nx, int ny, int nz, float dx, float dt, const float* ux0, const float* uy0, const float* uz0,
                     float* ux1, float* uy1, float* uz1, void* stream) {
    if (!dims_ok(nx, ny, nz) || !ux0 || !uy0 || !uz0 || !ux1 || !uy1 || !uz1) return EDGE_EINVAL;
    if (ux1 == ux0 || uy1 == uy0 || uz1 == uz0) return EDGE_EINVAL;
    const Mac mac = make_mac(ux0, uy0, uz0, nx, ny, nz, dx);
    const int g = grid_for(n_faces(nx, ny, nz), 128);
    if (mac.pow2) k_advect_sl<true><<<g, 128, 0, S(stream)>>>(mac, dt, ux1, uy1, uz1);
    else k_advect_sl<false><<<g, 128, 0, S(stream)>>>(mac, dt, ux1, uy1, uz1);
    return launch_status();
}

int edge_pullback_u(int nx, int ny, int nz, float dx, const float* ux0, const float* uy0, const float* uz0,
                    const float* posx, const float* posy, const float* posz, const float* colx, const float* coly,
                    const float* colz, const float* initx, const float* inity, const float* initz, float scale,
                    const float* subx, const float* suby, const float* subz, float* ux1, float* uy1, float* uz1,
                    void* stream) {
    if (!dims_ok(nx, ny, nz) || !ux0 || !uy0 || !uz0 || !posx || !posy || !posz || !colx || !coly || !colz || !ux1 ||
        !uy1 || !uz1)
        return EDGE_EINVAL;
    if (ux1 == ux0 || uy1 == uy0 || uz1 == uz0) return EDGE_EINVAL;
    Face3 pos = {{posx, posy, posz}}, col = {{colx, coly, colz}}, init = {{initx, inity, initz}},
          sub = {{subx, suby, subz}};
    const Mac mac = make_mac(ux0, uy0, uz0, nx, ny, nz, dx);
    const int g = grid_for(n_faces(nx, ny, nz));
    if (mac.pow2) k_pullback_u<true><<<g, kBlock, 0, S(stream)>>>(mac, pos, col, init, scale, sub, ux1, uy1, uz1);
    else k_pullback_u<false><<<g, kBlock, 0, S(stream)>>>(mac, pos, col, init, scale, sub, ux1, uy1, uz1);
    return launch_status();
}

int edge_map_u_psi(int variant, int nx, int ny, int nz, float dx, const float* ux0, const float* uy0,
                   const float* uz0, float* ux1, float* uy1, float* uz1, const float* psi, const float* Tx,
                   const float* Ty, const float* Tz, const float* dTx, const float* dTy, const float* dTz,
                   void* stream) {
    if (!dims_ok(nx, ny, nz) || !ux0 || !uy0 || !uz0 || !ux1 || !uy1 || !uz1 || !psi || !Tx || !Ty || !Tz)
        return EDGE_EINVAL;
    if (variant == HV_GARM && (!dTx || !dTy || !dTz)) return EDGE_EINVAL;
    if (ux1 == ux0 || uy1 == uy0 || uz1 == uz0) return EDGE_EINVAL;
    const float* T[3] = {Tx, Ty, Tz};
    const float* dT[3] = {dTx, dTy, dTz};
    MapF m = make_map(psi, T, dT, nullptr, nx, ny, nz, dx);
    Mac mac = make_mac(ux0, uy0, uz0, nx, ny, nz, dx);
    int g = grid_for(n_faces(nx, ny, nz), 128);
    if (variant == HV_FD) k_map_u_psi<HV_FD><<<g, 128, 0, S(stream)>>>(mac, m, ux1, uy1, uz1);
    else if (variant == HV_GARM) k_map_u_psi<HV_GARM><<<g, 128, 0, S(stream)>>>(mac, m, ux1, uy1, uz1);
    else return EDGE_EINVAL;
    return launch_status();
}

int edge_pullback_dye(int nx, int ny, int nz, float dx, const float* smoke0, const float* posx, const float* posy,
                      const float* posz, const float* init, float scale, const float* sub, const float* clampsrc,
                      int inplace_clamp, float* out, void* stream) {
    if (!dims_ok(nx, ny, nz) || !posx || !posy || !posz || !out) return EDGE_EINVAL;
    if (!inplace_clamp && !smoke0) return EDGE_EINVAL;
    if (inplace_clamp && !clampsrc) return EDGE_EINVAL;
    if (!al16(smoke0) || !al16(init) || !al16(sub) || !al16(clampsrc) || !al16(out)) return EDGE_EALIGN;
    if (!inplace_clamp && out == smoke0) return EDGE_EINVAL;
    Face3 pos = {{posx, posy, posz}};
    int n = nx * ny * nz;
    const Dye dye = make_dye(nx, ny, nz, dx);
    if (dye.pow2)
        k_pullback_dye<true><<<grid_for(n), kBlock, 0, S(stream)>>>(dye, smoke0, pos, init, scale, sub, clampsrc,
                                                                    inplace_clamp, out);
    else
        k_pullback_dye<false><<<grid_for(n), kBlock, 0, S(stream)>>>(dye, smoke0, pos, init, scale, sub, clampsrc,
                                                                     inplace_clamp, out);
    return launch_status();
}

int edge_smoke_psi(int variant, int mode, int nx, int ny, int nz, float dx, const float* smoke0, float* out,
                   const float* psi, const float* Tx, const float* Ty, const float* Tz, const float* dTx,
                   const float* dTy, const float* dTz, void* stream) {
    if (!dims_ok(nx, ny, nz) || !smoke0 || !out || !psi || !Tx || !Ty || !Tz || (mode != 0 && mode != 1))
        return EDGE_EINVAL;
    if (variant == HV_GARM && (!dTx || !dTy || !dTz)) return EDGE_EINVAL;
    if (!al16(smoke0) || !al16(out)) return EDGE_EALIGN;
    if (out == smoke0) return EDGE_EINVAL;
    const float* T[3] = {Tx, Ty, Tz};
    const float* dT[3] = {dTx, dTy, dTz};
    MapF m = make_map(psi, T, dT, nullptr, nx, ny, nz, dx);
    Dye d = make_dye(nx, ny, nz, dx);
    int g = grid_for(nx * ny * nz, 128);
    if (variant == HV_FD && mode == 0) k_smoke_psi<HV_FD, 0><<<g, 128, 0, S(stream)>>>(d, m, smoke0, out);
    else if (variant == HV_FD && mode == 1) k_smoke_psi<HV_FD, 1><<<g, 128, 0, S(stream)>>>(d, m, smoke0, out);
    else if (variant == HV_GARM && mode == 0) k_smoke_psi<HV_GARM, 0><<<g, 128, 0, S(stream)>>>(d, m, smoke0, out);
    else if (variant == HV_GARM && mode == 1) k_smoke_psi<HV_GARM, 1><<<g, 128, 0, S(stream)>>>(d, m, smoke0, out);
    else return EDGE_EINVAL;
    return launch_status();
}

int edge_clamp_u(int nx, int ny, int nz, const float* ux, const float* uy, const float* uz, const float* u1x,
                 const float* u1y, const float* u1z, float* u2x, float* u2y, float* u2z, void* stream) {
    if (!dims_ok(nx, ny, nz) || !ux || !uy || !uz || !u1x || !u1y || !u1z || !u2x || !u2y || !u2z) return EDGE_EINVAL;
    if (u2x == u1x || u2y == u1y || u2z == u1z) return EDGE_EINVAL;
    Face3 u = {{ux, uy, uz}}, u1 = {{u1x, u1y, u1z}};
    k_clamp_u<<<grid_for(n_faces(nx, ny, nz)), kBlock, 0, S(stream)>>>(nx, ny, nz, u, u1, u2x, u2y, u2z);
    return launch_status();
}

int edge_max_speed(int nx, int ny, int nz, const float* ux, const float* uy, const float* uz, float* out_max,
                   void* stream) {
    if (!dims_ok(nx, ny, nz) || !ux || !uy || !uz || !out_max) return EDGE_EINVAL;
    k_set_float<<<1, 1, 0, S(stream)>>>(out_max, 1.e-3f);
    int n = nx * ny * nz;
    int blocks = min(grid_for(n), 148 * 8);
    k_max_speed<<<blocks, kBlock, 0, S(stream)>>>(nx, ny, nz, ux, uy, uz, out_max);
    return launch_status();
}

int edge_compute_dt(const float* max_speed, float cfl, float dx, double visualize_dt, double* state, float* dt,
                    float* half_dt, void* stream) {
    if (!max_speed || !state || !dt || !half_dt) return EDGE_EINVAL;
    k_compute_dt<<<1, 1, 0, S(stream)>>>(max_speed, (double)cfl * (double)dx, visualize_dt, state, dt, half_dt);
    return launch_status();
}

int edge_axpy(long long n, const float* f1, const float* f2, float a, float* dest, void* stream) {
    if (n < 0 || (n && (!f1 || !dest))) return EDGE_EINVAL;
    if (n == 0) return EDGE_OK;
    int blocks = (int)std::min<long long>(grid_for(n), 148LL * 16);
    k_axpy<<<blocks, kBlock, 0, S(stream)>>>(n, f1, f2, a, dest);
    return launch_status();
}

int edge_copy(long long n, const float* src, float* dst, void* stream) {
    if (n < 0 || (n && (!src || !dst))) return EDGE_EINVAL;
    if (n == 0 || src == dst) return EDGE_OK;
    cudaError_t e = cudaMemcpyAsync(dst, src, (size_t)n * sizeof(float), cudaMemcpyDeviceToDevice, S(stream));
    return e == cudaSuccess ? EDGE_OK : (int)e;
}

int edge_add_vortex_ring(int nx, int ny, int nz, float dx, float w, float rad, float delta, const float* c,
                         const float* ex, const float* ey, float* u, float* smoke, const float* color,
                         int num_samples, void* stream) {
    if (!dims_ok(nx, ny, nz) || !c || !ex || !ey || !u || !smoke || !color || num_samples <= 0) return EDGE_EINVAL;
    Ring R;
    R.w = w; R.rad = rad; R.delta = delta; R.ns = num_samples;
    for (int a = 0; a < 3; a++) {
        R.c[a] = c[a]; R.ex[a] = ex[a]; R.ey[a] = ey[a]; R.color[a] = color[a];
    }
    k_vortex_ring<<<grid_for(nx * ny * nz), kBlock, 0, S(stream)>>>(nx, ny, nz, dx, R, u, smoke);
    return launch_status();
}

int edge_emit_smoke(int nx, int ny, int nz, float dx, const float* centers, const float* colors, int k, float radius,
                    float* smoke, void* stream) {
    if (!dims_ok(nx, ny, nz) || !centers || !colors || !smoke || k < 0 || k > 16) return EDGE_EINVAL;
    if (!al16(smoke)) return EDGE_EALIGN;
    Emitters E;
    E.k = k;
    E.radius = radius;
    for (int q = 0; q < k; q++) {
        for (int a = 0; a < 3; a++) E.c[q][a] = centers[3 * q + a];
        for (int a = 0; a < 4; a++) E.col[q][a] = colors[4 * q + a];
    }
    k_emit_spheres<<<grid_for(nx * ny * nz), kBlock, 0, S(stream)>>>(nx, ny, nz, dx, E, (float4*)smoke);
    return launch_status();
}

int edge_clamp_max(long long n, float hi, float* x, void* stream) {
    if (n < 0 || (n && !x)) return EDGE_EINVAL;
    if (n == 0) return EDGE_OK;
    int blocks = (int)std::min<long long>(grid_for(n), 148LL * 16);
    k_clamp_max<<<blocks, kBlock, 0, S(stream)>>>(n, hi, x);
    return launch_status();
}

int edge_split_central_vector(int nx, int ny, int nz, const float* vc, float* ux, float* uy, float* uz,
                              void* stream) {
    if (!dims_ok(nx, ny, nz) || !vc || !ux || !uy || !uz) return EDGE_EINVAL;
    k_split_central<<<grid_for(n_faces(nx, ny, nz)), kBlock, 0, S(stream)>>>(nx, ny, nz, vc, ux, uy, uz);
    return launch_status();
}

int edge_get_central_vector(int nx, int ny, int nz, const float* ux, const float* uy, const float* uz, float* vc,
                            void* stream) {
    if (!dims_ok(nx, ny, nz) || !vc || !ux || !uy || !uz) return EDGE_EINVAL;
    k_get_central<<<grid_for((long long)nx * ny * nz), kBlock, 0, S(stream)>>>(nx, ny, nz, ux, uy, uz, vc);
    return launch_status();
}

int edge_curl(int nx, int ny, int nz, float dx, const float* vf, float* cf, void* stream) {
    if (!dims_ok(nx, ny, nz) || !vf || !cf || vf == cf) return EDGE_EINVAL;
    k_curl<<<grid_for((long long)nx * ny * nz), kBlock, 0, S(stream)>>>(nx, ny, nz, dx, vf, cf);
    return launch_status();
}

}  // extern "C"
