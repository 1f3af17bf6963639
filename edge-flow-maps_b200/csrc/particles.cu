// Laden-particle kernels (sim/lp.py): grid-to-particle sampling with the
// quadratic B-spline MAC interpolant, the explicit particle update, the
// particle-to-grid drag scatter and the face-grid viscous Laplacian.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>

#include "edge_common.cuh"

using namespace edge;

namespace {

inline int grid_for(long long n, int b = 256) { return (int)((n + b - 1) / b); }
inline int st(void) {
    cudaError_t e = cudaPeekAtLastError();
    return e == cudaSuccess ? EDGE_OK : (int)e;
}
inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }
// EDGE_P2G_TILE=1: the shared-memory staged scatter; default: one global
// atomic per particle and tap
inline bool p2g_direct() {
    static const bool t = getenv("EDGE_P2G_TILE") && getenv("EDGE_P2G_TILE")[0] == '1';
    return !t;
}

// lp.py:6-29 update_particles_acc
__global__ void k_lp_acc(Mac mac, const float* __restrict__ vel, const float* __restrict__ pos, float* acc, int num,
                         int nmax, float dt, float St, float gravity) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nmax) return;
    float a[3] = {0.f, 0.f, 0.f};
    if (e < num) {
        float kk = 1.0f / St;
        float p[3] = {pos[3 * e], pos[3 * e + 1], pos[3 * e + 2]};
        float v[3], G[3][3];
        mac_sample<true>(mac, p, v, G);
        a[1] += gravity;
        for (int c = 0; c < 3; c++) a[c] -= kk * (vel[3 * e + c] - v[c]);
        for (int c = 0; c < 3; c++) a[c] /= (1.0f + kk * dt);
    }
    for (int c = 0; c < 3; c++) acc[3 * e + c] = a[c];
}

// lp.py:32-70 update_particles_velocity
__global__ void k_lp_velocity(const float* __restrict__ acc, float* vel, const float* __restrict__ pos, float dt,
                              float dx, int num, float Lx, float Ly, float Lz) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= num) return;
    float v[3], p[3] = {pos[3 * e], pos[3 * e + 1], pos[3 * e + 2]};
    for (int c = 0; c < 3; c++) v[c] = vel[3 * e + c] + acc[3 * e + c] * dt;
    if (p[1] < dx && v[1] < 0) v[1] = 0.0f;
    if (p[1] > Ly - 3 * dx && v[1] > 0) v[1] = 0.0f;
    if (p[0] < 3 * dx && v[0] < 0) v[0] = 0.0f;
    if (p[0] > Lx - 3 * dx && v[0] > 0) v[0] = 0.0f;
    if (p[2] < 3 * dx && v[2] < 0) v[2] = 0.0f;
    if (p[2] > Lz - 3 * dx && v[2] > 0) v[2] = 0.0f;
    for (int c = 0; c < 3; c++) vel[3 * e + c] = v[c];
}

// lp.py:73-97 calculate_velocity_diff
__global__ void k_lp_vel_diff(Mac mac, const float* __restrict__ vel, float* vdiff, const float* __restrict__ pos,
                              int num, float kk) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= num) return;
    float p[3] = {pos[3 * e], pos[3 * e + 1], pos[3 * e + 2]};
    float v[3], G[3][3];
    mac_sample<true>(mac, p, v, G);
    for (int c = 0; c < 3; c++) vdiff[3 * e + c] = kk * (vel[3 * e + c] - v[c]);
}

// lp.py:100-156 laden_particles_back_with_computing_particle: quadratic
// B-spline scatter of the drag onto the three face grids (atomic adds, like
// the reference's `+=` in a parallel loop)
__global__ void k_lp_p2g(int nx, int ny, int nz, float dx, float* dx_, float* dy_, float* dz_,
                         const float* __restrict__ vdiff, const float* __restrict__ pos,
                         const float* __restrict__ rad, int num, float lrad, float Lx, float Ly, float Lz) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= num) return;
    float p[3] = {pos[3 * e], pos[3 * e + 1], pos[3 * e + 2]};
    if (p[0] < 3 * dx || p[1] < 3 * dx || p[2] < 3 * dx || p[0] > Lx - 3 * dx || p[1] > Ly - 3 * dx ||
        p[2] > Lz - 3 * dx)
        return;
    float g[3] = {p[0] / dx, p[1] / dx, p[2] / dx};
    float r = rad[e];
    float scale = r * r * r / (lrad * lrad * lrad);
    float* D[3] = {dx_, dy_, dz_};
    for (int a = 0; a < 3; a++) {
        float off[3];
        int base[3];
        for (int c = 0; c < 3; c++) {
            off[c] = (c == a) ? 0.0f : 0.5f;
            base[c] = (int)(g[c] - off[c]);
        }
        int n0 = nx + (a == 0), n1 = ny + (a == 1), n2 = nz + (a == 2);
        float val = vdiff[3 * e + a];
        for (int oi = -1; oi < 3; oi++) {
            int f0 = base[0] + oi;
            if (f0 < 0 || f0 >= n0) continue;
            float wx = N2(g[0] - (float)f0 - off[0]);
            if (wx == 0.0f) continue;
            for (int oj = -1; oj < 3; oj++) {
                int f1 = base[1] + oj;
                if (f1 < 0 || f1 >= n1) continue;
                float wy = N2(g[1] - (float)f1 - off[1]);
                if (wy == 0.0f) continue;
                for (int ok = -1; ok < 3; ok++) {
                    int f2 = base[2] + ok;
                    if (f2 < 0 || f2 >= n2) continue;
                    float w = wx * wy * N2(g[2] - (float)f2 - off[2]);
                    if (w == 0.0f) continue;
                    atomicAdd(D[a] + idx3(f0, f1, f2, n1, n2), val * w * scale);
                }
            }
        }
    }
}

// The same scatter staged through shared memory.  A block takes 256
// consecutive particles; when the faces they touch (the bounding box of their
// 4x4x4 stencils, per face grid) fit the block's tile, the block accumulates
// there with shared-memory atomics and adds each touched face to the global
// grid once, instead of one global atomic per particle and tap (particles
// stored in cell order, as the workloads seed them, touch a few hundred faces
// per block; 256 x 81 taps otherwise).  A block whose particles are spread
// wider scatters directly.  Same weights and values as k_lp_p2g; only the
// order of the float additions differs (as between two runs of the atomic
// scatter).
constexpr int kP2GThreads = 256;
constexpr int kP2GTile = 10240;  // floats of shared memory per block (40 KB)

EDGE_D bool p2g_inside(const float (&p)[3], float dx, float Lx, float Ly, float Lz) {
    return !(p[0] < 3 * dx || p[1] < 3 * dx || p[2] < 3 * dx || p[0] > Lx - 3 * dx || p[1] > Ly - 3 * dx ||
             p[2] > Lz - 3 * dx);
}

__global__ void __launch_bounds__(kP2GThreads) k_lp_p2g_tile(int nx, int ny, int nz, float dx, float* dx_, float* dy_,
                                                             float* dz_, const float* __restrict__ vdiff,
                                                             const float* __restrict__ pos,
                                                             const float* __restrict__ rad, int num, float lrad,
                                                             float Lx, float Ly, float Lz) {
    __shared__ float tile[kP2GTile];
    __shared__ int lo_s[9], hi_s[9];
    __shared__ int use_tile;
    // the block's 256 particles are taken lane-major: lane l of warp w takes
    // particle 8 l + w, so the lanes of a warp hold particles 8 apart (in
    // the workloads' cell order, one per cell) and their taps hit a face of
    // the tile at most a few at a time, not all eight particles of a cell
    const int e = blockIdx.x * blockDim.x + (threadIdx.x & 31) * 8 + (threadIdx.x >> 5);
    float p[3] = {0.f, 0.f, 0.f};
    bool live = e < num;
    if (live) {
        p[0] = pos[3 * e];
        p[1] = pos[3 * e + 1];
        p[2] = pos[3 * e + 2];
        live = p2g_inside(p, dx, Lx, Ly, Lz);
    }
    const float g[3] = {p[0] / dx, p[1] / dx, p[2] / dx};
    // base index of each face grid's stencil (lp.py:130, 139, 148)
    int base[3][3];
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int c = 0; c < 3; c++) base[a][c] = (int)(g[c] - ((c == a) ? 0.0f : 0.5f));
    if (threadIdx.x < 9) {
        lo_s[threadIdx.x] = 0x7fffffff;
        hi_s[threadIdx.x] = -0x7fffffff;
    }
    __syncthreads();
    if (live) {
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int c = 0; c < 3; c++) {
                atomicMin(&lo_s[3 * a + c], base[a][c] - 1);
                atomicMax(&hi_s[3 * a + c], base[a][c] + 2);
            }
    }
    __syncthreads();
    // tile layout: face grid a occupies ext[a] = product of its box sides
    int off[4];
    int ext[3][3];
    off[0] = 0;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        long long v = 1;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            ext[a][c] = hi_s[3 * a + c] >= lo_s[3 * a + c] ? hi_s[3 * a + c] - lo_s[3 * a + c] + 1 : 0;
            v *= ext[a][c];
        }
        off[a + 1] = off[a] + (int)min(v, (long long)kP2GTile + 1);
    }
    if (threadIdx.x == 0) use_tile = off[3] <= kP2GTile;
    __syncthreads();
    const bool tiled = use_tile;
    if (tiled)
        for (int t = threadIdx.x; t < off[3]; t += blockDim.x) tile[t] = 0.0f;
    __syncthreads();
    if (live) {
        const float r = rad[e];
        const float scale = r * r * r / (lrad * lrad * lrad);
        float* D[3] = {dx_, dy_, dz_};
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const float offc[3] = {a == 0 ? 0.0f : 0.5f, a == 1 ? 0.0f : 0.5f, a == 2 ? 0.0f : 0.5f};
            const int n0 = nx + (a == 0), n1 = ny + (a == 1), n2 = nz + (a == 2);
            const float val = vdiff[3 * e + a];
            for (int oi = -1; oi < 3; oi++) {
                const int f0 = base[a][0] + oi;
                if (f0 < 0 || f0 >= n0) continue;
                const float wx = N2(g[0] - (float)f0 - offc[0]);
                if (wx == 0.0f) continue;
                for (int oj = -1; oj < 3; oj++) {
                    const int f1 = base[a][1] + oj;
                    if (f1 < 0 || f1 >= n1) continue;
                    const float wy = N2(g[1] - (float)f1 - offc[1]);
                    if (wy == 0.0f) continue;
                    for (int ok = -1; ok < 3; ok++) {
                        const int f2 = base[a][2] + ok;
                        if (f2 < 0 || f2 >= n2) continue;
                        const float w = wx * wy * N2(g[2] - (float)f2 - offc[2]);
                        if (w == 0.0f) continue;
                        const float add = val * w * scale;
                        if (tiled) {
                            const int t = off[a] + ((f0 - lo_s[3 * a]) * ext[a][1] + (f1 - lo_s[3 * a + 1])) * ext[a][2] +
                                          (f2 - lo_s[3 * a + 2]);
                            atomicAdd(&tile[t], add);
                        } else {
                            atomicAdd(D[a] + idx3(f0, f1, f2, n1, n2), add);
                        }
                    }
                }
            }
        }
    }
    if (!tiled) return;
    __syncthreads();
    float* D[3] = {dx_, dy_, dz_};
    for (int t = threadIdx.x; t < off[3]; t += blockDim.x) {
        const float v = tile[t];
        if (v == 0.0f) continue;
        const int a = t < off[1] ? 0 : (t < off[2] ? 1 : 2);
        int q = t - off[a];
        const int k = q % ext[a][2];
        q /= ext[a][2];
        const int j = q % ext[a][1];
        const int i = q / ext[a][1];
        const int n1 = ny + (a == 1), n2 = nz + (a == 2);
        atomicAdd(D[a] + idx3(lo_s[3 * a] + i, lo_s[3 * a + 1] + j, lo_s[3 * a + 2] + k, n1, n2), v);
    }
}

// lp.py:158-181 update_particles_position
__global__ void k_lp_position(const float* __restrict__ vel, float* pos, float dt, int num, float Lx, float Ly,
                              float Lz) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= num) return;
    float L[3] = {Lx, Ly, Lz};
    for (int c = 0; c < 3; c++) {
        float p = pos[3 * e + c] + vel[3 * e + c] * dt;
        if (p < 0) p = 0.0f;
        if (p > L[c]) p = L[c];
        pos[3 * e + c] = p;
    }
}

// lp.py:183-219 calculate_viscous_force on the three face grids
__global__ void k_lp_viscous(int nx, int ny, int nz, float dx, float nu, const float* __restrict__ ux,
                             const float* __restrict__ uy, const float* __restrict__ uz, float* vx, float* vy,
                             float* vz) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_faces(nx, ny, nz)) return;
    FaceIdx f = face_decompose(t, nx, ny, nz);
    int n0 = nx + (f.axis == 0), n1 = ny + (f.axis == 1), n2 = nz + (f.axis == 2);
    const float* u = f.axis == 0 ? ux : (f.axis == 1 ? uy : uz);
    float* o = f.axis == 0 ? vx : (f.axis == 1 ? vy : vz);
    auto s = [&](int i, int j, int k) {
        return __ldg(u + idx3(min(max(i, 0), n0 - 1), min(max(j, 0), n1 - 1), min(max(k, 0), n2 - 1), n1, n2));
    };
    int i = f.i, j = f.j, k = f.k;
    o[f.e] = nu * (s(i + 1, j, k) + s(i - 1, j, k) + s(i, j + 1, k) + s(i, j - 1, k) + s(i, j, k + 1) +
                   s(i, j, k - 1) + -6.0f * s(i, j, k)) / dx / dx;
}

// calc_max_particle_speed (run_edge.py:256-261): max |v| over the live
// particles, at least 1e-3 (bits of non-negative floats order as integers)
__global__ void k_lp_init_max(float* out) { *out = 1.0e-3f; }
__global__ void k_lp_max_speed(const float* __restrict__ vel, int num, float* out) {
    float best = 0.0f;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < num; e += gridDim.x * blockDim.x) {
        float a = vel[3 * e], b = vel[3 * e + 1], c = vel[3 * e + 2];
        best = fmaxf(best, sqrtf(a * a + b * b + c * c));
    }
    for (int o = 16; o > 0; o >>= 1) best = fmaxf(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0) atomicMax(reinterpret_cast<int*>(out), __float_as_int(best));
}

}  // namespace

extern "C" {

int edge_lp_max_speed(const float* vel, int num, float* out, void* stream) {
    if (num < 0 || !out || (num && !vel)) return EDGE_EINVAL;
    k_lp_init_max<<<1, 1, 0, S(stream)>>>(out);
    if (num > 0) k_lp_max_speed<<<std::min(grid_for(num), 148 * 8), 256, 0, S(stream)>>>(vel, num, out);
    return st();
}

int edge_lp_acc(int nx, int ny, int nz, float dx, const float* ux, const float* uy, const float* uz, const float* vel,
                const float* pos, float* acc, int num, int nmax, float dt, float St, float gravity, void* stream) {
    if (nx < 4 || ny < 4 || nz < 4 || !ux || !uy || !uz || num < 0 || nmax < num || (nmax && (!vel || !pos || !acc)))
        return EDGE_EINVAL;
    if (nmax == 0) return EDGE_OK;
    k_lp_acc<<<grid_for(nmax), 256, 0, S(stream)>>>(make_mac(ux, uy, uz, nx, ny, nz, dx), vel, pos, acc, num, nmax, dt,
                                                    St, gravity);
    return st();
}

int edge_lp_velocity(const float* acc, float* vel, const float* pos, float dt, float dx, int num, float Lx, float Ly,
                     float Lz, void* stream) {
    if (num < 0 || (num && (!acc || !vel || !pos))) return EDGE_EINVAL;
    if (num == 0) return EDGE_OK;
    k_lp_velocity<<<grid_for(num), 256, 0, S(stream)>>>(acc, vel, pos, dt, dx, num, Lx, Ly, Lz);
    return st();
}

int edge_lp_vel_diff(int nx, int ny, int nz, float dx, const float* ux, const float* uy, const float* uz,
                     const float* vel, float* vdiff, const float* pos, int num, float St, float density_ratio,
                     float epiral_radius_ratio, void* stream) {
    if (nx < 4 || ny < 4 || nz < 4 || !ux || !uy || !uz || num < 0 || (num && (!vel || !vdiff || !pos)))
        return EDGE_EINVAL;
    if (num == 0) return EDGE_OK;
    float eratio = 1.0f / (epiral_radius_ratio * epiral_radius_ratio * epiral_radius_ratio);
    float kk = 1.0f / St * density_ratio * eratio;
    k_lp_vel_diff<<<grid_for(num), 256, 0, S(stream)>>>(make_mac(ux, uy, uz, nx, ny, nz, dx), vel, vdiff, pos, num, kk);
    return st();
}

int edge_lp_p2g(int nx, int ny, int nz, float dx, float* dragx, float* dragy, float* dragz, const float* vdiff,
                const float* pos, const float* rad, int num, float laden_radius, float Lx, float Ly, float Lz,
                void* stream) {
    if (nx < 1 || ny < 1 || nz < 1 || !dragx || !dragy || !dragz || num < 0 || (num && (!vdiff || !pos || !rad)))
        return EDGE_EINVAL;
    cudaStream_t s = S(stream);
    cudaError_t e;
    if ((e = cudaMemsetAsync(dragx, 0, (size_t)(nx + 1) * ny * nz * 4, s)) != cudaSuccess) return (int)e;
    if ((e = cudaMemsetAsync(dragy, 0, (size_t)nx * (ny + 1) * nz * 4, s)) != cudaSuccess) return (int)e;
    if ((e = cudaMemsetAsync(dragz, 0, (size_t)nx * ny * (nz + 1) * 4, s)) != cudaSuccess) return (int)e;
    if (num == 0) return EDGE_OK;
    if (p2g_direct())
        k_lp_p2g<<<grid_for(num), 256, 0, s>>>(nx, ny, nz, dx, dragx, dragy, dragz, vdiff, pos, rad, num, laden_radius,
                                               Lx, Ly, Lz);
    else
        k_lp_p2g_tile<<<grid_for(num, kP2GThreads), kP2GThreads, 0, s>>>(nx, ny, nz, dx, dragx, dragy, dragz, vdiff,
                                                                          pos, rad, num, laden_radius, Lx, Ly, Lz);
    return st();
}

int edge_lp_position(const float* vel, float* pos, float dt, int num, float Lx, float Ly, float Lz, void* stream) {
    if (num < 0 || (num && (!vel || !pos))) return EDGE_EINVAL;
    if (num == 0) return EDGE_OK;
    k_lp_position<<<grid_for(num), 256, 0, S(stream)>>>(vel, pos, dt, num, Lx, Ly, Lz);
    return st();
}

int edge_lp_viscous(int nx, int ny, int nz, float dx, float Re, const float* ux, const float* uy, const float* uz,
                    float* visx, float* visy, float* visz, void* stream) {
    if (nx < 1 || ny < 1 || nz < 1 || !ux || !uy || !uz || !visx || !visy || !visz) return EDGE_EINVAL;
    k_lp_viscous<<<grid_for(n_faces(nx, ny, nz)), 256, 0, S(stream)>>>(nx, ny, nz, dx, 1.0f / Re, ux, uy, uz, visx,
                                                                       visy, visz);
    return st();
}

}  // extern "C"
