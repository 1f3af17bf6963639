// Laden-particle kernels (sim/lp.py): grid-to-particle sampling with the
// quadratic B-spline MAC interpolant, the explicit particle update, the
// particle-to-grid drag scatter and the face-grid viscous Laplacian.
#include <cuda_runtime.h>

#include <algorithm>

#include "edge_common.cuh"

using namespace edge;

namespace {

inline int grid_for(long long n, int b = 256) { return (int)((n + b - 1) / b); }
inline int st(void) {
    cudaError_t e = cudaPeekAtLastError();
    return e == cudaSuccess ? EDGE_OK : (int)e;
}
inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// lp.py:6-29 update_particles_acc
template <bool P2>
__global__ void k_lp_acc(Mac mac_, const float* __restrict__ vel, const float* __restrict__ pos, float* acc, int num,
                         int nmax, float dt, float St, float gravity) {
    const Mac mac = with_pow2<P2>(mac_);
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
template <bool P2>
__global__ void k_lp_vel_diff(Mac mac_, const float* __restrict__ vel, float* vdiff, const float* __restrict__ pos,
                              int num, float kk) {
    const Mac mac = with_pow2<P2>(mac_);
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
template <bool P2>
__global__ void k_lp_p2g(int nx, int ny, int nz, float dx, float inv_dx, float* dx_, float* dy_, float* dz_,
                         const float* __restrict__ vdiff, const float* __restrict__ pos,
                         const float* __restrict__ rad, int num, float lrad, float Lx, float Ly, float Lz) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= num) return;
    float p[3] = {pos[3 * e], pos[3 * e + 1], pos[3 * e + 2]};
    if (p[0] < 3 * dx || p[1] < 3 * dx || p[2] < 3 * dx || p[0] > Lx - 3 * dx || p[1] > Ly - 3 * dx ||
        p[2] > Lz - 3 * dx)
        return;
    float g[3] = {over_dx(p[0], dx, inv_dx, P2), over_dx(p[1], dx, inv_dx, P2), over_dx(p[2], dx, inv_dx, P2)};
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
        // the four taps' weights of each axis, once (the loops below used to
        // re-evaluate N2 for every tap of the inner loops)
        float W[3][4];
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
            for (int o = 0; o < 4; o++) W[c][o] = N2(g[c] - (float)(base[c] + o - 1) - off[c]);
#pragma unroll
        for (int oi = -1; oi < 3; oi++) {
            int f0 = base[0] + oi;
            if (f0 < 0 || f0 >= n0) continue;
            float wx = W[0][oi + 1];
            if (wx == 0.0f) continue;
#pragma unroll
            for (int oj = -1; oj < 3; oj++) {
                int f1 = base[1] + oj;
                if (f1 < 0 || f1 >= n1) continue;
                float wy = W[1][oj + 1];
                if (wy == 0.0f) continue;
#pragma unroll
                for (int ok = -1; ok < 3; ok++) {
                    int f2 = base[2] + ok;
                    if (f2 < 0 || f2 >= n2) continue;
                    float w = wx * wy * W[2][ok + 1];
                    if (w == 0.0f) continue;
                    atomicAdd(D[a] + idx3(f0, f1, f2, n1, n2), val * w * scale);
                }
            }
        }
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
    const Mac mac = make_mac(ux, uy, uz, nx, ny, nz, dx);
    if (mac.pow2) k_lp_acc<true><<<grid_for(nmax), 256, 0, S(stream)>>>(mac, vel, pos, acc, num, nmax, dt, St, gravity);
    else k_lp_acc<false><<<grid_for(nmax), 256, 0, S(stream)>>>(mac, vel, pos, acc, num, nmax, dt, St, gravity);
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
    const Mac mac = make_mac(ux, uy, uz, nx, ny, nz, dx);
    if (mac.pow2) k_lp_vel_diff<true><<<grid_for(num), 256, 0, S(stream)>>>(mac, vel, vdiff, pos, num, kk);
    else k_lp_vel_diff<false><<<grid_for(num), 256, 0, S(stream)>>>(mac, vel, vdiff, pos, num, kk);
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
    // p / dx as the reference writes it: the exact multiply by 1/dx when dx is a power of two
    if (pow2f(dx))
        k_lp_p2g<true><<<grid_for(num), 256, 0, s>>>(nx, ny, nz, dx, 1.0f / dx, dragx, dragy, dragz, vdiff, pos, rad,
                                                     num, laden_radius, Lx, Ly, Lz);
    else
        k_lp_p2g<false><<<grid_for(num), 256, 0, s>>>(nx, ny, nz, dx, 1.0f / dx, dragx, dragy, dragz, vdiff, pos, rad,
                                                      num, laden_radius, Lx, Ly, Lz);
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
