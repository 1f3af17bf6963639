// MGPCG pressure projection (sim/mgpcg.py, sim/mgpcg_solid.py) for sm_100a.
//
// One solve is a CUDA graph: set-up kernels, then a conditional WHILE node
// whose body is one CG iteration, then the pressure-gradient update.  The CG
// scalars (alpha, beta, r.r, z.r, the recentering mean) live in device memory
// and are produced by "last block" reductions (per-block float64 partials
// summed in block order, so results are run-to-run deterministic); the body's
// last kernel sets the loop condition, so a solve makes no host round trip.
//
// Arrays: level l holds r[l], z[l] (float32, n>>l per axis); the fine level
// also holds x, two p buffers (ping-pong, so update_p fuses into the Ap
// stencil) and Ap.  The all-Neumann recentering (mgpcg.py:169-175) is kept as
// a pending scalar `mean` that every reader of r[0] subtracts, and that the
// r update folds into the stored residual.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <tuple>
#include <vector>

#include "edge_common.cuh"

using namespace edge;

namespace {

enum { ST_RUNNING = 0, ST_CONVERGED = 1, ST_NOCONV = 2, ST_NAN = 3 };

struct SolveState {
    double zTr, pAp, rTr, rsum, tol, abs_tol, rel_tol, div_sum;
    float alpha, beta, mean, pad0;
    int it, max_iters, status, setup;
    int pcur, all_neumann, n_fluid, pad1;
    unsigned int counter[8];
    unsigned long long kernels;  // kernels of this solver run so far (launch accounting)
};

constexpr size_t kCoarseSmem = 160 * 1024;  // shared memory for the coarse group

struct Lvl {
    int n0, n1, n2;
    float* r;
    float* z;
    const int* bm;  // solid mask (level 0: the caller's; NULL: plain solver)
};

struct Ctx {  // everything a kernel needs, passed by value
    Lvl lv[16];
    int L;
    int bt[6];
    float* x;
    float* p[2];
    float* Ap;
    float* div;
    double* partials;
    SolveState* st;
    cudaGraphConditionalHandle cond;
    int use_cond;  // 0: kernels run outside a graph (eager mode), no loop condition
    int lc;        // first level of the shared-memory coarse group (k_coarse)
    int cmoff;     // float offset of the coarse group's masks in shared memory
    int csmem;     // dynamic shared memory of k_coarse (bytes)
};

EDGE_D void set_cond(const Ctx& c, unsigned v) {
    if (c.use_cond) cudaGraphSetConditional(c.cond, v);
}

EDGE_D bool is_fluid(const int* bm, int e) { return bm == nullptr || __ldg(bm + e) <= 0; }

// mgpcg.py:100-110 num_fluid_neighbors (+ mgpcg_solid.py:113-130 solid faces)
EDGE_D float n_fluid(const Ctx& c, const Lvl& L, int i, int j, int k) {
    float num = 6.0f;
    int I[3] = {i, j, k}, D[3] = {L.n0, L.n1, L.n2};
#pragma unroll
    for (int a = 0; a < 3; a++) {
        if (I[a] <= 0 && c.bt[2 * a] == 2) num -= 1.0f;
        else if (L.bm && I[a] > 0) {
            int e = idx3(i - (a == 0), j - (a == 1), k - (a == 2), L.n1, L.n2);
            if (__ldg(L.bm + e) > 0) num -= 1.0f;
        }
        if (I[a] >= D[a] - 1 && c.bt[2 * a + 1] == 2) num -= 1.0f;
        else if (L.bm && I[a] < D[a] - 1) {
            int e = idx3(i + (a == 0), j + (a == 1), k + (a == 2), L.n1, L.n2);
            if (__ldg(L.bm + e) > 0) num -= 1.0f;
        }
    }
    return num;
}

// ---------------------------------------------------------------------------
// reductions
// ---------------------------------------------------------------------------
template <int N>
EDGE_D void block_sum(double (&v)[N]) {
    __shared__ double sm[N][32];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < N; q++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
    }
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < N; q++) sm[q][wid] = v[q];
    __syncthreads();
    int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int q = 0; q < N; q++) {
        double t = (wid == 0 && lane < nw) ? sm[q][lane] : 0.0;
        if (wid == 0)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        v[q] = t;  // valid in thread 0
    }
}

// Publish this block's partials; returns true in every thread of the block
// that arrives last, after which partials[q*nblk + b] hold all blocks' sums.
template <int N>
EDGE_D bool last_block(const Ctx& c, int slot, double (&v)[N]) {
    __shared__ bool am_last;
    block_sum<N>(v);
    int nblk = gridDim.x * gridDim.y * gridDim.z;
    int b = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < N; q++) c.partials[q * nblk + b] = v[q];
        __threadfence();
        unsigned t = atomicAdd(&c.st->counter[slot], 1u);
        am_last = (t == (unsigned)nblk - 1);
    }
    __syncthreads();
    return am_last;
}

// Sum the published partials (fixed order: deterministic) in the last block.
template <int N>
EDGE_D void final_sum(const Ctx& c, int slot, double (&out)[N]) {
    __threadfence();
    int nblk = gridDim.x * gridDim.y * gridDim.z;
    double v[N];
#pragma unroll
    for (int q = 0; q < N; q++) {
        double s = 0.0;
        for (int b = threadIdx.x; b < nblk; b += blockDim.x) s += __ldcg(c.partials + q * nblk + b);
        v[q] = s;
    }
    block_sum<N>(v);
#pragma unroll
    for (int q = 0; q < N; q++) out[q] = v[q];
    if (threadIdx.x == 0) c.st->counter[slot] = 0;
}

EDGE_D bool running(const Ctx& c) { return *((volatile int*)&c.st->status) == ST_RUNNING; }

// every solver kernel counts itself once (block 0, thread 0), including the
// ones that return early once the loop has finished
EDGE_D void count_launch(SolveState* st) {
    if (blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0) atomicAdd(&st->kernels, 1ull);
}

// ---------------------------------------------------------------------------
// set-up: apply_bc, divergence, solid correction, recentering mean
// ---------------------------------------------------------------------------
struct Faces {
    float* u[3];
    float* f[3];
};

// mgpcg.py:374-392 apply_bc (walls)
__global__ void k_apply_walls(Ctx c, int nx, int ny, int nz, Faces U) {
    count_launch(c.st);
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_faces(nx, ny, nz)) return;
    FaceIdx f = face_decompose(t, nx, ny, nz);
    int I[3] = {f.i, f.j, f.k};
    int D[3] = {nx, ny, nz};
    int a = f.axis;
    if ((I[a] == 0 && c.bt[2 * a] == 2) || (I[a] == D[a] && c.bt[2 * a + 1] == 2)) U.u[a][f.e] = 0.0f;
}

// mgpcg_solid.py:344-356: solid-cell velocities on their six faces
__global__ void k_apply_solid(SolveState* st, int nx, int ny, int nz, const int* bm, const float* bvel, Faces U) {
    count_launch(st);
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nx * ny * nz || bm[e] <= 0) return;
    int k = e % nz, j = (e / nz) % ny, i = e / (ny * nz);
    float vx = bvel[3 * e], vy = bvel[3 * e + 1], vz = bvel[3 * e + 2];
    U.u[0][idx3(i, j, k, ny, nz)] = vx;
    U.u[0][idx3(i + 1, j, k, ny, nz)] = vx;
    U.u[1][idx3(i, j, k, ny + 1, nz)] = vy;
    U.u[1][idx3(i, j + 1, k, ny + 1, nz)] = vy;
    U.u[2][idx3(i, j, k, ny, nz + 1)] = vz;
    U.u[2][idx3(i, j, k + 1, ny, nz + 1)] = vz;
}

// mgpcg.py:394-404 divergence + init(u_div, -1) (mgpcg.py:67-75); solid:
// mgpcg_solid.py:359-372 (fluid-only divergence, its sum and count).  With
// rhs != NULL the right-hand side is taken from rhs instead (edge_mgpcg_solve).
__global__ void k_setup_rhs(Ctx c, Faces U, const float* rhs, double abs_tol, double rel_tol, int max_iters) {
    count_launch(c.st);
    const Lvl& L = c.lv[0];
    int n = L.n0 * L.n1 * L.n2;
    double v[3] = {0.0, 0.0, 0.0};  // sum div (fluid), fluid count, sum r
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        int k = e % L.n2, j = (e / L.n2) % L.n1, i = e / (L.n1 * L.n2);
        float d;
        bool fl = is_fluid(L.bm, e);
        if (rhs) {
            d = -rhs[e];
        } else if (fl) {
            const int nx = L.n0, ny = L.n1, nz = L.n2;
            float vl = U.u[0][idx3(i, j, k, ny, nz)], vr = U.u[0][idx3(i + 1, j, k, ny, nz)];
            float vb = U.u[1][idx3(i, j, k, ny + 1, nz)], vt = U.u[1][idx3(i, j + 1, k, ny + 1, nz)];
            float va = U.u[2][idx3(i, j, k, ny, nz + 1)], vc = U.u[2][idx3(i, j, k + 1, ny, nz + 1)];
            d = vr - vl + vt - vb + vc - va;
            (void)nx;
        } else {
            d = 0.0f;
        }
        c.div[e] = d;
        float r = d * -1.0f;
        L.r[e] = r;
        c.x[e] = 0.0f;
        c.p[0][e] = 0.0f;
        c.p[1][e] = 0.0f;
        if (fl) {
            v[0] += d;
            v[1] += 1.0;
        }
        v[2] += r;
    }
    if (last_block<3>(c, 0, v)) {
        double s[3];
        final_sum<3>(c, 0, s);
        if (threadIdx.x == 0) {
            SolveState* st = c.st;
            st->div_sum = (double)(float)s[0];
            st->n_fluid = (int)s[1];
            st->rsum = s[2];
            st->abs_tol = abs_tol;
            st->rel_tol = rel_tol;
            st->max_iters = max_iters;
            st->it = 0;
            st->status = ST_RUNNING;
            st->setup = 1;
            st->beta = 0.0f;
            st->alpha = 0.0f;
            st->pcur = 0;
            st->mean = st->all_neumann ? (float)(s[2] / (double)n) : 0.0f;
        }
    }
}

// mgpcg_solid.py:374-383, 422-424: if the fluid divergence sums to > 0,
// subtract its mean from every fluid cell; then the recentering mean.
__global__ void k_solid_fix(Ctx c) {
    count_launch(c.st);
    const Lvl& L = c.lv[0];
    int n = L.n0 * L.n1 * L.n2;
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    SolveState* st = c.st;
    float dsum = (float)st->div_sum;
    bool fix = dsum > 0.0f && st->n_fluid > 0;
    float avg = fix ? dsum / (float)st->n_fluid : 0.0f;
    double v[1] = {0.0};
    for (; e < n; e += gridDim.x * blockDim.x) {
        float r = L.r[e];
        if (fix && is_fluid(L.bm, e)) {
            float d = c.div[e] - avg;
            c.div[e] = d;
            r = d * -1.0f;
            L.r[e] = r;
        }
        v[0] += r;
    }
    if (last_block<1>(c, 1, v)) {
        double s[1];
        final_sum<1>(c, 1, s);
        if (threadIdx.x == 0) st->mean = st->all_neumann ? (float)(s[0] / (double)n) : 0.0f;
    }
}

// mgpcg_solid.py:87-97 downsample_bm: coarse solid iff all 8 children solid
__global__ void k_downsample_bm(SolveState* st, const int* fine, int* coarse, int c0, int c1, int c2, int f1, int f2) {
    count_launch(st);
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= c0 * c1 * c2) return;
    int K = e % c2, J = (e / c2) % c1, I = e / (c1 * c2);
    int all = 1;
    for (int a = 0; a < 2; a++)
        for (int b = 0; b < 2; b++)
            for (int q = 0; q < 2; q++)
                if (fine[idx3(2 * I + a, 2 * J + b, 2 * K + q, f1, f2)] <= 0) all = 0;
    coarse[e] = all;
}

// ---------------------------------------------------------------------------
// CG vector kernels
// ---------------------------------------------------------------------------
// update_p (mgpcg.py:143-145) fused into compute_Ap (mgpcg.py:112-117):
// p_new = z + beta p_old on the fly (also at the stencil neighbours), Ap,
// and the p.Ap partials; the last block forms alpha (mgpcg.py:237-240).
__global__ void __launch_bounds__(256) k_cg_ap(Ctx c) {
    count_launch(c.st);
    // The loop stops unless the iteration's last kernel completes its
    // reduction and asks to continue: a lost reduction can never spin.
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        set_cond(c, 0);
        if (c.st->it > c.st->max_iters + 8) c.st->status = ST_NOCONV;  // hard cap
    }
    if (!running(c)) return;
    const Lvl& L = c.lv[0];
    const int n = L.n0 * L.n1 * L.n2;
    SolveState* st = c.st;
    const int pc = st->pcur;
    const float* __restrict__ po = c.p[pc];
    float* __restrict__ pn = c.p[pc ^ 1];
    const float* __restrict__ z = L.z;
    const float beta = st->beta;
    const int s0 = L.n1 * L.n2, s1 = L.n2;
    double v[1] = {0.0};
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        float pe = 0.0f, ape = 0.0f;
        if (is_fluid(L.bm, e)) {
            int k = e % L.n2, j = (e / L.n2) % L.n1, i = e / s0;
            pe = __ldg(z + e) + beta * __ldg(po + e);
            float nsum = 0.0f;
            if (i < L.n0 - 1 && is_fluid(L.bm, e + s0)) nsum += __ldg(z + e + s0) + beta * __ldg(po + e + s0);
            if (i > 0 && is_fluid(L.bm, e - s0)) nsum += __ldg(z + e - s0) + beta * __ldg(po + e - s0);
            if (j < L.n1 - 1 && is_fluid(L.bm, e + s1)) nsum += __ldg(z + e + s1) + beta * __ldg(po + e + s1);
            if (j > 0 && is_fluid(L.bm, e - s1)) nsum += __ldg(z + e - s1) + beta * __ldg(po + e - s1);
            if (k < L.n2 - 1 && is_fluid(L.bm, e + 1)) nsum += __ldg(z + e + 1) + beta * __ldg(po + e + 1);
            if (k > 0 && is_fluid(L.bm, e - 1)) nsum += __ldg(z + e - 1) + beta * __ldg(po + e - 1);
            ape = n_fluid(c, L, i, j, k) * pe - nsum;
            v[0] += (double)pe * (double)ape;
        }
        pn[e] = pe;
        c.Ap[e] = ape;
    }
    if (last_block<1>(c, 2, v)) {
        double sm[1];
        final_sum<1>(c, 2, sm);
        if (threadIdx.x == 0) {
            double pAp = (double)(float)sm[0];
            st->pAp = pAp;
            st->alpha = (float)(st->zTr / (pAp + 1e-12));
            st->pcur = pc ^ 1;
        }
    }
}

// update_x / update_r (mgpcg.py:133-141), r.r (mgpcg.py:247-249), the
// convergence test (mgpcg.py:254) and the recentering sum (mgpcg.py:169-175).
// Solid cells only take the recentering (mgpcg_solid.py:197-202).
__global__ void __launch_bounds__(256) k_cg_xr(Ctx c) {
    count_launch(c.st);
    if (!running(c)) return;
    const Lvl& L = c.lv[0];
    int n = L.n0 * L.n1 * L.n2;
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    SolveState* st = c.st;
    float alpha = st->alpha, mean = st->mean;
    const float* __restrict__ p = c.p[st->pcur];
    double v[2] = {0.0, 0.0};
    for (; e < n; e += gridDim.x * blockDim.x) {
        float r = L.r[e] - mean;
        if (is_fluid(L.bm, e)) {
            c.x[e] += alpha * __ldg(p + e);
            r -= alpha * __ldg(c.Ap + e);
            v[0] += (double)r * (double)r;
        }
        L.r[e] = r;
        v[1] += r;
    }
    if (last_block<2>(c, 3, v)) {
        double s[2];
        final_sum<2>(c, 3, s);
        if (threadIdx.x == 0) {
            double rTr = (double)(float)s[0];
            st->rTr = rTr;
            st->rsum = s[1];
            st->mean = st->all_neumann ? (float)(s[1] / (double)n) : 0.0f;
            if (!(rTr == rTr) || rTr > 1e300) st->status = ST_NAN;
            else if (rTr < st->tol) st->status = ST_CONVERGED;
        }
    }
}

// ---------------------------------------------------------------------------
// V-cycle (mgpcg.py:177-195)
// ---------------------------------------------------------------------------
// Red-black Gauss-Seidel (mgpcg.py:160-167) runs as half sweeps: a half sweep
// of colour c updates the cells with (i+j+k)&1 == c and reads only cells of
// the other colour, so no update depends on another in the same launch, and a
// cell's own old value is never read.  Hence:
//   * z = 0 before the first down sweep needs no fill (that half sweep reads
//     nothing, mode HS_FIRST);
//   * the prolongation z[l] += z[l+1][I/2] (mgpcg.py:155-158) that precedes
//     the up sweeps is applied on the fly to the neighbours the first up half
//     sweep reads (mode HS_PROLONG): every cell is overwritten by a half sweep
//     before its own value is read again, and solid cells are never read.
// Levels with more cells than fit in shared memory use one thread per pair
// of cells along k (the pair holds one cell of each colour); the remaining
// coarse levels run as one thread block in shared memory (k_coarse).
enum { HS_FIRST = 0, HS_PLAIN = 1, HS_PROLONG = 2, HS_ZR = 3 };

EDGE_D float nb_val(const Lvl& L, const Lvl* C, int e, int i, int j, int k, bool prolong) {
    float v = __ldg(L.z + e);
    if (prolong) v += __ldg(C->z + idx3(i >> 1, j >> 1, k >> 1, C->n1, C->n2));
    return v;
}

template <int MODE>
__global__ void __launch_bounds__(256) k_hsweep(Ctx c, int l, int color) {
    count_launch(c.st);
    if (!running(c)) {
        if (MODE == HS_ZR && blockIdx.x == 0 && threadIdx.x == 0) set_cond(c, 0);
        return;
    }
    const Lvl& L = c.lv[l];
    const Lvl* C = MODE == HS_PROLONG ? &c.lv[l + 1] : nullptr;
    const float mean = l == 0 ? c.st->mean : 0.0f;
    const int h2 = L.n2 >> 1;
    const int npair = L.n0 * L.n1 * h2;
    double v[1] = {0.0};
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < npair; t += gridDim.x * blockDim.x) {
        int kk = t % h2, r = t / h2;
        int j = r % L.n1, i = r / L.n1;
        int k = 2 * kk + ((i + j + color) & 1);
        int e = idx3(i, j, k, L.n1, L.n2);
        const int s1 = L.n2, s0 = L.n1 * L.n2;
        float rv = __ldg(L.r + e) - mean;
        float zn = 0.0f;
        if (is_fluid(L.bm, e)) {
            float ns = 0.0f;
            if (MODE != HS_FIRST) {
                const bool pr = MODE == HS_PROLONG;
                if (k < L.n2 - 1 && is_fluid(L.bm, e + 1)) ns += nb_val(L, C, e + 1, i, j, k + 1, pr);
                if (k > 0 && is_fluid(L.bm, e - 1)) ns += nb_val(L, C, e - 1, i, j, k - 1, pr);
                if (j < L.n1 - 1 && is_fluid(L.bm, e + s1)) ns += nb_val(L, C, e + s1, i, j + 1, k, pr);
                if (j > 0 && is_fluid(L.bm, e - s1)) ns += nb_val(L, C, e - s1, i, j - 1, k, pr);
                if (i < L.n0 - 1 && is_fluid(L.bm, e + s0)) ns += nb_val(L, C, e + s0, i + 1, j, k, pr);
                if (i > 0 && is_fluid(L.bm, e - s0)) ns += nb_val(L, C, e - s0, i - 1, j, k, pr);
            }
            // neighbour_sum order differs from the reference's (+x,-x,+y,...):
            // a rounding-level difference
            zn = (rv + ns) / n_fluid(c, L, i, j, k);
            L.z[e] = zn;
            if (MODE == HS_ZR) v[0] += (double)zn * (double)rv;
        }
        if (MODE == HS_ZR) {
            // the other cell of the pair (final from the previous half sweep)
            int kp = k ^ 1;
            int ep = idx3(i, j, kp, L.n1, L.n2);
            if (is_fluid(L.bm, ep)) v[0] += (double)__ldg(L.z + ep) * (double)(__ldg(L.r + ep) - mean);
        }
    }
    if (MODE == HS_ZR) {
        // mgpcg.py:263-275: z.r, beta, update bookkeeping, loop condition
        if (last_block<1>(c, 4, v)) {
            double sm[1];
            final_sum<1>(c, 4, sm);
            if (threadIdx.x == 0) {
                SolveState* st = c.st;
                double zTr = (double)(float)sm[0];
                if (st->setup) {
                    st->setup = 0;
                    st->zTr = zTr;
                    st->beta = 0.0f;
                    st->tol = fmax(st->abs_tol, zTr * st->rel_tol);
                    if (st->max_iters <= 0) st->status = ST_NOCONV;
                } else {
                    st->beta = (float)(zTr / (st->zTr + 1e-12));
                    st->zTr = zTr;
                    st->it += 1;
                    if (st->it >= st->max_iters) st->status = ST_NOCONV;
                }
                set_cond(c, st->status == ST_RUNNING ? 1u : 0u);
            }
        }
    }
}

// restrict (mgpcg.py:147-153): r[l+1] = sum over the 8 children of
// (r - A z) / (dim - 1), solid children skipped (mgpcg_solid.py:168-174)
__global__ void __launch_bounds__(256) k_restrict(Ctx c, int l) {
    count_launch(c.st);
    if (!running(c)) return;
    const Lvl& L = c.lv[l];
    const Lvl& C = c.lv[l + 1];
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= C.n0 * C.n1 * C.n2) return;
    const float mean = l == 0 ? c.st->mean : 0.0f;
    int K = e % C.n2, J = (e / C.n2) % C.n1, I = e / (C.n1 * C.n2);
    const float* __restrict__ z = L.z;
    float acc = 0.0f;
    int stride[3] = {L.n1 * L.n2, L.n2, 1};
    for (int a = 0; a < 2; a++)
        for (int b = 0; b < 2; b++)
            for (int q = 0; q < 2; q++) {
                int i = 2 * I + a, j = 2 * J + b, k = 2 * K + q;
                int f = idx3(i, j, k, L.n1, L.n2);
                if (!is_fluid(L.bm, f)) continue;
                int Ix[3] = {i, j, k}, D[3] = {L.n0, L.n1, L.n2};
                float ns = 0.0f;
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    if (Ix[d] < D[d] - 1 && is_fluid(L.bm, f + stride[d])) ns += __ldg(z + f + stride[d]);
                    if (Ix[d] > 0 && is_fluid(L.bm, f - stride[d])) ns += __ldg(z + f - stride[d]);
                }
                float res = (__ldg(L.r + f) - mean) - (n_fluid(c, L, i, j, k) * __ldg(z + f) - ns);
                acc += res * 0.5f;
            }
    C.r[e] = acc;
}

// The coarse levels lc..L-1 of a V-cycle in one thread block out of shared
// memory: down sweeps + restriction, 20 bottom sweeps, prolongation + up
// sweeps (mgpcg.py:177-195); z[lc] is written back for the prolongation into
// level lc-1.  With ZR (the whole grid fits, lc == 0) it also forms z.r and
// runs the end-of-iteration bookkeeping.
struct CoarseLvl {
    int n0, n1, n2, off;  // off: float offset of r (z follows) in shared memory
};
EDGE_D bool c_fluid(const unsigned char* bm, int e) { return bm == nullptr || bm[e] == 0; }

template <bool ZR>
__global__ void __launch_bounds__(1024) k_coarse(Ctx c, int lc, int moff) {
    extern __shared__ float sh[];
    count_launch(c.st);
    if (!running(c)) {
        if (ZR && threadIdx.x == 0) set_cond(c, 0);
        return;
    }
    const int L = c.L;
    const bool solid = c.lv[0].bm != nullptr;
    unsigned char* bmall = reinterpret_cast<unsigned char*>(sh + moff);
    const float mean = lc == 0 ? c.st->mean : 0.0f;
    // layout
    CoarseLvl cl[16];
    int off = 0, boff = 0, bo[16];
    for (int l = lc; l < L; l++) {
        cl[l].n0 = c.lv[l].n0; cl[l].n1 = c.lv[l].n1; cl[l].n2 = c.lv[l].n2;
        cl[l].off = off;
        int n = cl[l].n0 * cl[l].n1 * cl[l].n2;
        off += 2 * n;
        bo[l] = boff;
        boff += n;
    }
    // load r[lc] and the masks
    {
        int n = cl[lc].n0 * cl[lc].n1 * cl[lc].n2;
        for (int e = threadIdx.x; e < n; e += blockDim.x) sh[cl[lc].off + e] = __ldg(c.lv[lc].r + e) - mean;
        if (solid)
            for (int l = lc; l < L; l++) {
                int m = cl[l].n0 * cl[l].n1 * cl[l].n2;
                for (int e = threadIdx.x; e < m; e += blockDim.x) bmall[bo[l] + e] = __ldg(c.lv[l].bm + e) > 0;
            }
    }
    __syncthreads();
    auto half = [&](int l, int color, int mode) {
        // mode: 0 from zero, 1 plain, 2 with the prolongation of l+1
        const CoarseLvl& q = cl[l];
        float* r = sh + q.off;
        float* z = r + q.n0 * q.n1 * q.n2;
        const unsigned char* bm = solid ? bmall + bo[l] : nullptr;
        const float* zc = mode == 2 ? sh + cl[l + 1].off + cl[l + 1].n0 * cl[l + 1].n1 * cl[l + 1].n2 : nullptr;
        int n = q.n0 * q.n1 * q.n2;
        for (int e = threadIdx.x; e < n; e += blockDim.x) {
            int k = e % q.n2, j = (e / q.n2) % q.n1, i = e / (q.n1 * q.n2);
            if (((i + j + k) & 1) != color || !c_fluid(bm, e)) continue;
            float ns = 0.0f;
            if (mode != 0) {
                int I[3] = {i, j, k}, D[3] = {q.n0, q.n1, q.n2}, S[3] = {q.n1 * q.n2, q.n2, 1};
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    for (int sgn = -1; sgn <= 1; sgn += 2) {
                        int ni = I[a] + sgn;
                        if (ni < 0 || ni >= D[a]) continue;
                        int f = e + sgn * S[a];
                        if (!c_fluid(bm, f)) continue;
                        float v = z[f];
                        if (mode == 2) {
                            int J[3] = {i, j, k};
                            J[a] = ni;
                            const CoarseLvl& u = cl[l + 1];
                            v += zc[((J[0] >> 1) * u.n1 + (J[1] >> 1)) * u.n2 + (J[2] >> 1)];
                        }
                        ns += v;
                    }
                }
            }
            // num_fluid_neighbors (mgpcg.py:100-110 / mgpcg_solid.py:113-130)
            float num = 6.0f;
            {
                int I[3] = {i, j, k}, D[3] = {q.n0, q.n1, q.n2}, S[3] = {q.n1 * q.n2, q.n2, 1};
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    if (I[a] <= 0 && c.bt[2 * a] == 2) num -= 1.0f;
                    else if (bm && I[a] > 0 && bm[e - S[a]]) num -= 1.0f;
                    if (I[a] >= D[a] - 1 && c.bt[2 * a + 1] == 2) num -= 1.0f;
                    else if (bm && I[a] < D[a] - 1 && bm[e + S[a]]) num -= 1.0f;
                }
            }
            z[e] = (r[e] + ns) / num;
        }
        __syncthreads();
    };
    // down
    for (int l = lc; l < L - 1; l++) {
        half(l, 0, 0);
        half(l, 1, 1);
        half(l, 0, 1);
        half(l, 1, 1);
        // restrict into r[l+1]
        const CoarseLvl& q = cl[l];
        const CoarseLvl& u = cl[l + 1];
        float* r = sh + q.off;
        float* z = r + q.n0 * q.n1 * q.n2;
        float* rc = sh + u.off;
        const unsigned char* bm = solid ? bmall + bo[l] : nullptr;
        int m = u.n0 * u.n1 * u.n2;
        for (int ce = threadIdx.x; ce < m; ce += blockDim.x) {
            int K = ce % u.n2, J = (ce / u.n2) % u.n1, I = ce / (u.n1 * u.n2);
            float acc = 0.0f;
            for (int a = 0; a < 2; a++)
                for (int b = 0; b < 2; b++)
                    for (int cc = 0; cc < 2; cc++) {
                        int i = 2 * I + a, j = 2 * J + b, k = 2 * K + cc;
                        int e = (i * q.n1 + j) * q.n2 + k;
                        if (!c_fluid(bm, e)) continue;
                        int Ix[3] = {i, j, k}, D[3] = {q.n0, q.n1, q.n2}, S[3] = {q.n1 * q.n2, q.n2, 1};
                        float ns = 0.0f, num = 6.0f;
                        for (int d = 0; d < 3; d++) {
                            if (Ix[d] < D[d] - 1 && c_fluid(bm, e + S[d])) ns += z[e + S[d]];
                            if (Ix[d] > 0 && c_fluid(bm, e - S[d])) ns += z[e - S[d]];
                            if (Ix[d] <= 0 && c.bt[2 * d] == 2) num -= 1.0f;
                            else if (bm && Ix[d] > 0 && bm[e - S[d]]) num -= 1.0f;
                            if (Ix[d] >= D[d] - 1 && c.bt[2 * d + 1] == 2) num -= 1.0f;
                            else if (bm && Ix[d] < D[d] - 1 && bm[e + S[d]]) num -= 1.0f;
                        }
                        float res = r[e] - (num * z[e] - ns);
                        acc += res * 0.5f;
                    }
            rc[ce] = acc;
        }
        __syncthreads();
    }
    // bottom (mgpcg.py:186-189)
    half(L - 1, 0, 0);
    half(L - 1, 1, 1);
    for (int it = 1; it < 20; it++) {
        half(L - 1, 0, 1);
        half(L - 1, 1, 1);
    }
    // up
    for (int l = L - 2; l >= lc; l--) {
        half(l, 1, 2);
        half(l, 0, 1);
        half(l, 1, 1);
        half(l, 0, 1);
    }
    // write back z[lc] (solid cells keep their last value, never read)
    {
        const CoarseLvl& q = cl[lc];
        int n = q.n0 * q.n1 * q.n2;
        const float* z = sh + q.off + n;
        for (int e = threadIdx.x; e < n; e += blockDim.x) c.lv[lc].z[e] = z[e];
    }
    if (ZR) {
        const CoarseLvl& q = cl[lc];
        int n = q.n0 * q.n1 * q.n2;
        const float* r = sh + q.off;
        const float* z = r + n;
        double v[1] = {0.0};
        for (int e = threadIdx.x; e < n; e += blockDim.x)
            if (c_fluid(solid ? bmall + bo[lc] : nullptr, e)) v[0] += (double)z[e] * (double)r[e];
        block_sum<1>(v);
        if (threadIdx.x == 0) {
            SolveState* st = c.st;
            double zTr = (double)(float)v[0];
            if (st->setup) {
                st->setup = 0;
                st->zTr = zTr;
                st->beta = 0.0f;
                st->tol = fmax(st->abs_tol, zTr * st->rel_tol);
                if (st->max_iters <= 0) st->status = ST_NOCONV;
            } else {
                st->beta = (float)(zTr / (st->zTr + 1e-12));
                st->zTr = zTr;
                st->it += 1;
                if (st->it >= st->max_iters) st->status = ST_NOCONV;
            }
            set_cond(c, st->status == ST_RUNNING ? 1u : 0u);
        }
    }
}

// mgpcg.py:406-432 subtract_grad_p (p = x, get_result mgpcg.py:77-85) + the
// wall part of the final apply_bc; Poisson_with_buffer's force (mgpcg.py:448-479)
__global__ void k_grad_p(Ctx c, int nx, int ny, int nz, Faces U) {
    count_launch(c.st);
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_faces(nx, ny, nz)) return;
    FaceIdx f = face_decompose(t, nx, ny, nz);
    int a = f.axis;
    int I[3] = {f.i, f.j, f.k}, D[3] = {nx, ny, nz};
    int hi[3] = {min(f.i, nx - 1), min(f.j, ny - 1), min(f.k, nz - 1)};
    int lo[3] = {hi[0], hi[1], hi[2]};
    lo[a] = max(I[a] - 1, 0);
    float pr = c.x[idx3(hi[0], hi[1], hi[2], ny, nz)];
    float pl = c.x[idx3(lo[0], lo[1], lo[2], ny, nz)];
    if (I[a] - 1 < 0) pl = 0.0f;
    if (I[a] >= D[a]) pr = 0.0f;
    float g = pr - pl;
    float u = U.u[a][f.e] - g;
    if ((I[a] == 0 && c.bt[2 * a] == 2) || (I[a] == D[a] && c.bt[2 * a + 1] == 2)) u = 0.0f;
    U.u[a][f.e] = u;
    if (U.f[a]) U.f[a][f.e] = -g;
}

__global__ void k_copy(SolveState* st, const float* a, float* b, int n) {
    if (st) count_launch(st);
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n) b[e] = a[e];
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
inline int grid_for(long long n, int b = 256) { return (int)((n + b - 1) / b); }

inline int cu(cudaError_t e) { return e == cudaSuccess ? EDGE_OK : (int)e; }
#define CK(x)                        \
    do {                             \
        int _r = cu(x);              \
        if (_r != EDGE_OK) return _r; \
    } while (0)

struct GraphKey {
    const void* a[7];
    double abs_tol, rel_tol;
    int max_iters;
    bool operator<(const GraphKey& o) const {
        return std::tie(a[0], a[1], a[2], a[3], a[4], a[5], a[6], abs_tol, rel_tol, max_iters) <
               std::tie(o.a[0], o.a[1], o.a[2], o.a[3], o.a[4], o.a[5], o.a[6], o.abs_tol, o.rel_tol, o.max_iters);
    }
};

struct Solver {
    Ctx ctx;
    int nx, ny, nz;
    bool solid;
    const float* bvel;
    int precision;
    std::vector<void*> allocs;
    std::map<GraphKey, cudaGraphExec_t> graphs;
    std::vector<cudaGraph_t> graph_defs;
    SolveState* st_host;  // pinned
    int max_blocks;
};

int alloc(Solver* s, void** p, size_t bytes) {
    CK(cudaMalloc(p, bytes));
    s->allocs.push_back(*p);
    return EDGE_OK;
}

// The levels lc..L-1 that fit in kCoarseSmem of shared memory together go to
// k_coarse; the finer ones run half-sweep kernels.
void plan_coarse(Ctx& c, bool solid) {
    for (int lc = 0; lc < c.L; lc++) {
        size_t floats = 0, cells = 0;
        for (int l = lc; l < c.L; l++) {
            size_t n = (size_t)c.lv[l].n0 * c.lv[l].n1 * c.lv[l].n2;
            floats += 2 * n;
            cells += n;
        }
        size_t bytes = floats * sizeof(float) + (solid ? cells : 0) + 16;
        if (bytes <= kCoarseSmem || lc == c.L - 1) {
            c.lc = lc;
            c.cmoff = (int)floats;
            c.csmem = (int)bytes;
            return;
        }
    }
}

int prepare_coarse_kernels(const Ctx& c) {
    if ((size_t)c.csmem > kCoarseSmem) return EDGE_EINVAL;  // the coarsest level alone must fit
    if (c.csmem > 48 * 1024) {
        CK(cudaFuncSetAttribute(k_coarse<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, c.csmem));
        CK(cudaFuncSetAttribute(k_coarse<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, c.csmem));
    }
    return EDGE_OK;
}

// One V-cycle (mgpcg.py:177-195); with final_zr the last kernel also forms
// z.r and the end-of-iteration bookkeeping (mgpcg.py:263-277).
// reduction and sweep kernels loop over their cells with at most this many
// blocks (8 per SM), which bounds the last-block atomics
constexpr int kMaxBlocks = 148 * 8;
inline int rgrid(long long n) { return (int)std::min<long long>(grid_for(n), kMaxBlocks); }

void enqueue_vcycle_ctx(const Ctx& c, cudaStream_t stream, bool final_zr) {
    const int lc = c.lc;
    for (int l = 0; l < lc; l++) {
        const Lvl& L = c.lv[l];
        int g = rgrid((long long)L.n0 * L.n1 * (L.n2 / 2));
        k_hsweep<HS_FIRST><<<g, 256, 0, stream>>>(c, l, 0);
        k_hsweep<HS_PLAIN><<<g, 256, 0, stream>>>(c, l, 1);
        k_hsweep<HS_PLAIN><<<g, 256, 0, stream>>>(c, l, 0);
        k_hsweep<HS_PLAIN><<<g, 256, 0, stream>>>(c, l, 1);
        const Lvl& C = c.lv[l + 1];
        k_restrict<<<grid_for((long long)C.n0 * C.n1 * C.n2), 256, 0, stream>>>(c, l);
    }
    if (final_zr && lc == 0) k_coarse<true><<<1, 1024, c.csmem, stream>>>(c, lc, c.cmoff);
    else k_coarse<false><<<1, 1024, c.csmem, stream>>>(c, lc, c.cmoff);
    for (int l = lc - 1; l >= 0; l--) {
        const Lvl& L = c.lv[l];
        int g = rgrid((long long)L.n0 * L.n1 * (L.n2 / 2));
        k_hsweep<HS_PROLONG><<<g, 256, 0, stream>>>(c, l, 1);
        k_hsweep<HS_PLAIN><<<g, 256, 0, stream>>>(c, l, 0);
        k_hsweep<HS_PLAIN><<<g, 256, 0, stream>>>(c, l, 1);
        if (l == 0 && final_zr) k_hsweep<HS_ZR><<<g, 256, 0, stream>>>(c, l, 0);
        else k_hsweep<HS_PLAIN><<<g, 256, 0, stream>>>(c, l, 0);
    }
}

void enqueue_vcycle(Solver* s, cudaStream_t stream, bool final_zr) { enqueue_vcycle_ctx(s->ctx, stream, final_zr); }

// The body of one CG iteration (mgpcg.py:236-277), enqueued on `stream`.
void enqueue_iteration(Solver* s, cudaStream_t stream) {
    Ctx& c = s->ctx;
    int n = c.lv[0].n0 * c.lv[0].n1 * c.lv[0].n2;
    k_cg_ap<<<rgrid(n), 256, 0, stream>>>(c);
    k_cg_xr<<<rgrid(n), 256, 0, stream>>>(c);
    enqueue_vcycle(s, stream, true);
}

// set-up kernels of Poisson / solve, then the conditional while node, then
// the gradient update; captured into a graph
int build_graph(Solver* s, Faces U, const float* rhs, float* xout, double abs_tol, double rel_tol, int max_iters,
                cudaGraphExec_t* exec) {
    cudaStream_t cs;
    CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t graph;
    CK(cudaGraphCreate(&graph, 0));
    cudaGraphConditionalHandle handle;
    CK(cudaGraphConditionalHandleCreate(&handle, graph, 0, cudaGraphCondAssignDefault));
    s->ctx.cond = handle;
    s->ctx.use_cond = 1;
    Ctx& c = s->ctx;
    int n = c.lv[0].n0 * c.lv[0].n1 * c.lv[0].n2;
    int nx = s->nx, ny = s->ny, nz = s->nz;
    // 1) set-up
    CK(cudaStreamBeginCaptureToGraph(cs, graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    if (!rhs) {
        k_apply_walls<<<grid_for(n_faces(nx, ny, nz)), 256, 0, cs>>>(c, nx, ny, nz, U);
        if (s->solid) k_apply_solid<<<grid_for(n), 256, 0, cs>>>(c.st, nx, ny, nz, c.lv[0].bm, s->bvel, U);
    }
    if (s->solid) {
        for (int l = 1; l < c.L; l++) {
            const Lvl& F = c.lv[l - 1];
            const Lvl& C = c.lv[l];
            k_downsample_bm<<<grid_for((long long)C.n0 * C.n1 * C.n2), 256, 0, cs>>>(c.st, F.bm, (int*)C.bm, C.n0, C.n1,
                                                                                    C.n2, F.n1, F.n2);
        }
    }
    CK(cudaMemsetAsync(c.st->counter, 0, sizeof(c.st->counter), cs));  // fresh reduction counters
    k_setup_rhs<<<rgrid(n), 256, 0, cs>>>(c, U, rhs, abs_tol, rel_tol, max_iters);
    if (s->solid && !rhs) k_solid_fix<<<rgrid(n), 256, 0, cs>>>(c);
    enqueue_vcycle(s, cs, true);  // first preconditioner application + z.r + tol
    cudaGraph_t g2;
    CK(cudaStreamEndCapture(cs, &g2));
    // leaf of the set-up chain
    size_t nn = 0;
    CK(cudaGraphGetNodes(graph, nullptr, &nn));
    std::vector<cudaGraphNode_t> nodes(nn);
    CK(cudaGraphGetNodes(graph, nodes.data(), &nn));
    cudaGraphNode_t leaf = nullptr;
    for (auto nd : nodes) {
        size_t nout = 0;
        CK(cudaGraphNodeGetDependentNodes(nd, nullptr, &nout));
        if (nout == 0) leaf = nd;
    }
    // 2) while (condition) { one CG iteration }
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t cnode;
    CK(cudaGraphAddNode(&cnode, graph, &leaf, 1, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    CK(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    enqueue_iteration(s, cs);
    cudaGraph_t b2;
    CK(cudaStreamEndCapture(cs, &b2));
    // 3) finish
    CK(cudaStreamBeginCaptureToGraph(cs, graph, &cnode, nullptr, 1, cudaStreamCaptureModeThreadLocal));
    if (!rhs) {
        k_grad_p<<<grid_for(n_faces(nx, ny, nz)), 256, 0, cs>>>(c, nx, ny, nz, U);
        if (s->solid) k_apply_solid<<<grid_for(n), 256, 0, cs>>>(c.st, nx, ny, nz, c.lv[0].bm, s->bvel, U);
    } else {
        k_copy<<<grid_for(n), 256, 0, cs>>>(c.st, c.x, xout, n);
    }
    CK(cudaStreamEndCapture(cs, &g2));
    int r = cu(cudaGraphInstantiate(exec, graph, 0));
    s->graph_defs.push_back(graph);
    cudaStreamDestroy(cs);
    return r;
}

// The same kernels driven by a host loop (one status read per iteration, as
// the reference does); selected with EDGE_MGPCG_EAGER=1 for profiling tools
// that replay kernels one by one.
int run_solve_eager(Solver* s, Faces U, const float* rhs, float* xout, double abs_tol, double rel_tol, int max_iters,
                    cudaStream_t cs) {
    s->ctx.use_cond = 0;
    Ctx& c = s->ctx;
    int n = c.lv[0].n0 * c.lv[0].n1 * c.lv[0].n2;
    int nx = s->nx, ny = s->ny, nz = s->nz;
    if (!rhs) {
        k_apply_walls<<<grid_for(n_faces(nx, ny, nz)), 256, 0, cs>>>(c, nx, ny, nz, U);
        if (s->solid) k_apply_solid<<<grid_for(n), 256, 0, cs>>>(c.st, nx, ny, nz, c.lv[0].bm, s->bvel, U);
    }
    if (s->solid)
        for (int l = 1; l < c.L; l++) {
            const Lvl& F = c.lv[l - 1];
            const Lvl& C = c.lv[l];
            k_downsample_bm<<<grid_for((long long)C.n0 * C.n1 * C.n2), 256, 0, cs>>>(c.st, F.bm, (int*)C.bm, C.n0,
                                                                                    C.n1, C.n2, F.n1, F.n2);
        }
    CK(cudaMemsetAsync(c.st->counter, 0, sizeof(c.st->counter), cs));
    k_setup_rhs<<<rgrid(n), 256, 0, cs>>>(c, U, rhs, abs_tol, rel_tol, max_iters);
    if (s->solid && !rhs) k_solid_fix<<<rgrid(n), 256, 0, cs>>>(c);
    enqueue_vcycle(s, cs, true);
    for (int it = 0; it <= max_iters + 8; it++) {
        CK(cudaMemcpyAsync(&s->st_host->status, &c.st->status, sizeof(int), cudaMemcpyDeviceToHost, cs));
        CK(cudaStreamSynchronize(cs));
        if (s->st_host->status != ST_RUNNING) break;
        enqueue_iteration(s, cs);
    }
    if (!rhs) {
        k_grad_p<<<grid_for(n_faces(nx, ny, nz)), 256, 0, cs>>>(c, nx, ny, nz, U);
        if (s->solid) k_apply_solid<<<grid_for(n), 256, 0, cs>>>(c.st, nx, ny, nz, c.lv[0].bm, s->bvel, U);
    } else {
        k_copy<<<grid_for(n), 256, 0, cs>>>(c.st, c.x, xout, n);
    }
    return cu(cudaPeekAtLastError());
}

int run_solve(Solver* s, Faces U, const float* rhs, float* xout, double abs_tol, double rel_tol, int max_iters,
              cudaStream_t stream) {
    static const bool eager = getenv("EDGE_MGPCG_EAGER") && getenv("EDGE_MGPCG_EAGER")[0] == '1';
    if (eager) return run_solve_eager(s, U, rhs, xout, abs_tol, rel_tol, max_iters, stream);
    GraphKey key;
    memset(&key, 0, sizeof(key));
    key.a[0] = U.u[0]; key.a[1] = U.u[1]; key.a[2] = U.u[2];
    key.a[3] = U.f[0]; key.a[4] = U.f[1]; key.a[5] = U.f[2];
    key.a[6] = rhs ? (const void*)rhs : (const void*)xout;
    key.abs_tol = abs_tol; key.rel_tol = rel_tol; key.max_iters = max_iters;
    auto it = s->graphs.find(key);
    cudaGraphExec_t exec;
    if (it == s->graphs.end()) {
        int r = build_graph(s, U, rhs, xout, abs_tol, rel_tol, max_iters, &exec);
        if (r != EDGE_OK) return r;
        s->graphs[key] = exec;
    } else {
        exec = it->second;
    }
    return cu(cudaGraphLaunch(exec, stream));
}

}  // namespace

extern "C" {

int edge_mgpcg_create(void** handle, int nx, int ny, int nz, int base_level, const int* bt, const int* mask,
                      const float* bvel, int precision) {
    if (!handle || !bt || nx < 2 || ny < 2 || nz < 2) return EDGE_EINVAL;
    if ((mask == nullptr) != (bvel == nullptr)) return EDGE_EINVAL;
    if (precision != 0) return EDGE_EINVAL;
    long long n = (long long)nx * ny * nz;
    if (n * 3 >= (1LL << 31)) return EDGE_EINVAL;
    int mn = std::min(nx, std::min(ny, nz));
    int lg = 0;
    while ((1 << (lg + 1)) <= mn) lg++;
    int L = lg - base_level + 1;  // mgpcg.py:34
    if (L < 1 || L > 16) return EDGE_EINVAL;
    for (int l = 1; l < L; l++) {
        int f = 1 << l;
        // restrict writes r[l+1][I//2]: every level must halve exactly
        if (nx % f || ny % f || nz % f) return EDGE_EINVAL;
    }
    Solver* s = new Solver();
    s->nx = nx; s->ny = ny; s->nz = nz;
    s->solid = mask != nullptr;
    s->bvel = bvel;
    s->precision = precision;
    Ctx& c = s->ctx;
    memset(&c, 0, sizeof(c));
    c.L = L;
    for (int q = 0; q < 6; q++) c.bt[q] = bt[q];
    int r = EDGE_OK;
    for (int l = 0; l < L && r == EDGE_OK; l++) {
        Lvl& V = c.lv[l];
        V.n0 = nx >> l; V.n1 = ny >> l; V.n2 = nz >> l;
        size_t m = (size_t)V.n0 * V.n1 * V.n2;
        r = alloc(s, (void**)&V.r, m * sizeof(float));
        if (r == EDGE_OK) r = alloc(s, (void**)&V.z, m * sizeof(float));
        if (r == EDGE_OK) r = cu(cudaMemset(V.z, 0, m * sizeof(float)));
        if (s->solid) {
            if (l == 0) V.bm = mask;
            else if (r == EDGE_OK) r = alloc(s, (void**)&V.bm, m * sizeof(int));
        }
    }
    plan_coarse(c, s->solid);
    if (r == EDGE_OK) r = prepare_coarse_kernels(c);
    if (r == EDGE_OK) r = alloc(s, (void**)&c.x, n * sizeof(float));
    if (r == EDGE_OK) r = alloc(s, (void**)&c.p[0], n * sizeof(float));
    if (r == EDGE_OK) r = alloc(s, (void**)&c.p[1], n * sizeof(float));
    if (r == EDGE_OK) r = alloc(s, (void**)&c.Ap, n * sizeof(float));
    if (r == EDGE_OK) r = alloc(s, (void**)&c.div, n * sizeof(float));
    long long maxblk = std::max<long long>(grid_for(n), grid_for(n_faces(nx, ny, nz))) + 1024;
    if (r == EDGE_OK) r = alloc(s, (void**)&c.partials, 3 * maxblk * sizeof(double));
    if (r == EDGE_OK) r = alloc(s, (void**)&c.st, sizeof(SolveState));
    if (r == EDGE_OK) {
        SolveState st;
        memset(&st, 0, sizeof(st));
        st.all_neumann = (bt[0] + bt[1] + bt[2] + bt[3] + bt[4] + bt[5]) == 12;
        r = cu(cudaMemcpy(c.st, &st, sizeof(st), cudaMemcpyHostToDevice));
    }
    if (r == EDGE_OK) r = cu(cudaMallocHost((void**)&s->st_host, sizeof(SolveState)));
    if (r != EDGE_OK) {
        for (void* p : s->allocs) cudaFree(p);
        delete s;
        return r;
    }
    *handle = s;
    return EDGE_OK;
}

int edge_mgpcg_destroy(void* handle) {
    if (!handle) return EDGE_EINVAL;
    Solver* s = (Solver*)handle;
    cudaDeviceSynchronize();
    for (auto& kv : s->graphs) cudaGraphExecDestroy(kv.second);
    for (auto g : s->graph_defs) cudaGraphDestroy(g);
    for (void* p : s->allocs) cudaFree(p);
    cudaFreeHost(s->st_host);
    delete s;
    return EDGE_OK;
}

int edge_mgpcg_levels(void* handle) { return handle ? ((Solver*)handle)->ctx.L : EDGE_EINVAL; }

int edge_mgpcg_kernel_count(void* handle, long long* count, void* stream) {
    if (!handle || !count) return EDGE_EINVAL;
    Solver* s = (Solver*)handle;
    CK(cudaMemcpyAsync(s->st_host, s->ctx.st, sizeof(SolveState), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    CK(cudaStreamSynchronize((cudaStream_t)stream));
    *count = (long long)s->st_host->kernels;
    return EDGE_OK;
}

int edge_mgpcg_poisson(void* handle, float* ux, float* uy, float* uz, float* fx, float* fy, float* fz,
                       double abs_tol, double rel_tol, int max_iters, void* stream) {
    if (!handle || !ux || !uy || !uz) return EDGE_EINVAL;
    if ((fx == nullptr) != (fy == nullptr) || (fx == nullptr) != (fz == nullptr)) return EDGE_EINVAL;
    Solver* s = (Solver*)handle;
    if (max_iters < 0) max_iters = s->solid ? 100 : 400;
    Faces U = {{ux, uy, uz}, {fx, fy, fz}};
    return run_solve(s, U, nullptr, nullptr, abs_tol, rel_tol, max_iters, (cudaStream_t)stream);
}

int edge_mgpcg_solve(void* handle, const float* b, float* x, double abs_tol, double rel_tol, int max_iters,
                     void* stream) {
    if (!handle || !b || !x) return EDGE_EINVAL;
    Solver* s = (Solver*)handle;
    if (max_iters < 0) max_iters = s->solid ? 100 : 400;
    Faces U = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
    return run_solve(s, U, b, x, abs_tol, rel_tol, max_iters, (cudaStream_t)stream);
}

int edge_mgpcg_result(void* handle, int* iters, double* rTr, int* status, void* stream) {
    if (!handle) return EDGE_EINVAL;
    Solver* s = (Solver*)handle;
    CK(cudaMemcpyAsync(s->st_host, s->ctx.st, sizeof(SolveState), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    CK(cudaStreamSynchronize((cudaStream_t)stream));
    const SolveState& st = *s->st_host;
    if (iters) *iters = st.it;
    if (rTr) *rTr = st.rTr;
    if (status)
        *status = st.status == ST_CONVERGED ? EDGE_OK : (st.status == ST_NAN ? EDGE_ENAN : EDGE_ENOCONV);
    return EDGE_OK;
}

int edge_mgpcg_vcycle(void* handle, const float* r, float* z, void* stream) {
    if (!handle || !r || !z) return EDGE_EINVAL;
    Solver* s = (Solver*)handle;
    cudaStream_t st = (cudaStream_t)stream;
    Ctx c = s->ctx;
    int n = c.lv[0].n0 * c.lv[0].n1 * c.lv[0].n2;
    // status = running, mean = 0, setup flag off so the z.r epilogue is inert
    SolveState* hs = s->st_host;
    CK(cudaMemcpyAsync(hs, c.st, sizeof(SolveState), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    hs->status = ST_RUNNING;
    hs->mean = 0.0f;
    hs->setup = 1;
    hs->max_iters = 1;
    hs->abs_tol = 0.0;
    hs->rel_tol = 0.0;
    CK(cudaMemcpyAsync(c.st, hs, sizeof(SolveState), cudaMemcpyHostToDevice, st));
    k_copy<<<grid_for(n), 256, 0, st>>>(nullptr, r, c.lv[0].r, n);
    // outside a graph there is no loop condition to set
    c.use_cond = 0;
    enqueue_vcycle_ctx(c, st, false);
    k_copy<<<grid_for(n), 256, 0, st>>>(nullptr, c.lv[0].z, z, n);
    return cu(cudaPeekAtLastError());
}

__global__ void k_apply_A(Ctx c, const float* p, float* Ap) {
    const Lvl& L = c.lv[0];
    int n = L.n0 * L.n1 * L.n2;
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    if (!is_fluid(L.bm, e)) { Ap[e] = 0.0f; return; }
    int k = e % L.n2, j = (e / L.n2) % L.n1, i = e / (L.n1 * L.n2);
    int I[3] = {i, j, k}, D[3] = {L.n0, L.n1, L.n2};
    int stride[3] = {L.n1 * L.n2, L.n2, 1};
    float ns = 0.0f;
    for (int a = 0; a < 3; a++) {
        if (I[a] < D[a] - 1 && is_fluid(L.bm, e + stride[a])) ns += p[e + stride[a]];
        if (I[a] > 0 && is_fluid(L.bm, e - stride[a])) ns += p[e - stride[a]];
    }
    Ap[e] = n_fluid(c, L, i, j, k) * p[e] - ns;
}

int edge_mgpcg_apply_A(void* handle, const float* p, float* Ap, void* stream) {
    if (!handle || !p || !Ap) return EDGE_EINVAL;
    Solver* s = (Solver*)handle;
    const Lvl& L = s->ctx.lv[0];
    k_apply_A<<<grid_for((long long)L.n0 * L.n1 * L.n2), 256, 0, (cudaStream_t)stream>>>(s->ctx, p, Ap);
    return cu(cudaPeekAtLastError());
}

int edge_mgpcg_get(void* handle, int which, float* dst, void* stream) {
    if (!handle || !dst) return EDGE_EINVAL;
    Solver* s = (Solver*)handle;
    const Lvl& L = s->ctx.lv[0];
    size_t n = (size_t)L.n0 * L.n1 * L.n2;
    const float* src = which == 0 ? s->ctx.div : (which == 1 ? s->ctx.x : nullptr);
    if (!src) return EDGE_EINVAL;
    return cu(cudaMemcpyAsync(dst, src, n * sizeof(float), cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
}

}  // extern "C"

// ===========================================================================
// Projection without any device allocation
// ===========================================================================
// For callers that cannot allocate device memory while they run: code
// embedded in another runtime that owns the whole device heap (a host
// framework with its own caching allocator, or a CUDA-graph-replaying engine
// that forbids cudaMalloc after warm-up), or a plugin that is handed only its
// input/output buffers.  The solver's scratch (level pyramid, CG vectors,
// reduction partials, loop state) lives in file-scope __device__ arrays sized
// for at most 262144 cells (64^3); every GPU that loads the library holds them
// (about 8 MB) until the process exits.  Solves run on the host-driven loop
// (one status read per iteration, as the reference's solve does).
namespace {

constexpr long long kNoAllocMaxCells = 262144;  // 64^3 cells
constexpr long long kNoAllocFloats = 7 * kNoAllocMaxCells + kNoAllocMaxCells / 2 + 4096;
constexpr int kNoAllocMaxBlocks = 4096;

static __device__ __align__(256) float g_noalloc_scratch[kNoAllocFloats];
static __device__ __align__(256) double g_noalloc_partials[3 * kNoAllocMaxBlocks];
static __device__ __align__(256) SolveState g_noalloc_state;

struct NoAllocAddrs {
    float* scratch;
    double* partials;
    SolveState* state;
    bool ready;
};
constexpr int kMaxDevices = 64;
NoAllocAddrs g_noalloc_addrs[kMaxDevices];

// Host code may not use the arrays' names as device addresses: resolve them
// once per device (with that device current).
int noalloc_addrs(NoAllocAddrs** out) {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return EDGE_EINVAL;
    NoAllocAddrs& a = g_noalloc_addrs[dev];
    if (!a.ready) {
        CK(cudaGetSymbolAddress((void**)&a.scratch, g_noalloc_scratch));
        CK(cudaGetSymbolAddress((void**)&a.partials, g_noalloc_partials));
        CK(cudaGetSymbolAddress((void**)&a.state, g_noalloc_state));
        a.ready = true;
    }
    *out = &a;
    return EDGE_OK;
}

}  // namespace

extern "C" int edge_mgpcg_poisson_noalloc(int nx, int ny, int nz, int base_level, const int* bt, float* ux, float* uy,
                                          float* uz, double abs_tol, double rel_tol, int max_iters, int* iters,
                                          double* rTr, int* status, void* stream) {
    if (!bt || !ux || !uy || !uz || nx < 2 || ny < 2 || nz < 2) return EDGE_EINVAL;
    long long n = (long long)nx * ny * nz;
    if (n > kNoAllocMaxCells) return EDGE_EINVAL;  // beyond the static scratch
    int mn = std::min(nx, std::min(ny, nz));
    int lg = 0;
    while ((1 << (lg + 1)) <= mn) lg++;
    int L = lg - base_level + 1;  // mgpcg.py:34
    if (L < 1 || L > 16) return EDGE_EINVAL;
    for (int l = 1; l < L; l++)
        if (nx % (1 << l) || ny % (1 << l) || nz % (1 << l)) return EDGE_EINVAL;
    if ((n + 255) / 256 > kNoAllocMaxBlocks) return EDGE_EINVAL;
    if (max_iters < 0) max_iters = 400;
    NoAllocAddrs* A = nullptr;
    int r = noalloc_addrs(&A);
    if (r != EDGE_OK) return r;
    cudaStream_t cs = (cudaStream_t)stream;
    // carve the scratch: 256-byte aligned slices
    Solver s;  // host-side description only; its containers stay empty
    s.nx = nx; s.ny = ny; s.nz = nz;
    s.solid = false;
    s.bvel = nullptr;
    s.precision = 0;
    s.st_host = nullptr;
    Ctx& c = s.ctx;
    memset(&c, 0, sizeof(c));
    c.L = L;
    for (int q = 0; q < 6; q++) c.bt[q] = bt[q];
    long long off = 0;
    auto take = [&](long long count) {
        float* p = A->scratch + off;
        off += (count + 63) / 64 * 64;
        return p;
    };
    for (int l = 0; l < L; l++) {
        Lvl& V = c.lv[l];
        V.n0 = nx >> l; V.n1 = ny >> l; V.n2 = nz >> l;
        long long m = (long long)V.n0 * V.n1 * V.n2;
        V.r = take(m);
        V.z = take(m);
        V.bm = nullptr;
    }
    c.x = take(n);
    c.p[0] = take(n);
    c.p[1] = take(n);
    c.Ap = take(n);
    c.div = take(n);
    if (off > kNoAllocFloats) return EDGE_EINVAL;
    c.partials = A->partials;
    c.st = A->state;
    c.use_cond = 0;
    plan_coarse(c, false);
    r = prepare_coarse_kernels(c);
    if (r != EDGE_OK) return r;
    // the loop state starts clean on every call (the arrays keep the last
    // call's contents); x and p are zeroed by the set-up kernel
    SolveState init;
    memset(&init, 0, sizeof(init));
    init.all_neumann = (bt[0] + bt[1] + bt[2] + bt[3] + bt[4] + bt[5]) == 12;
    CK(cudaMemcpyAsync(c.st, &init, sizeof(init), cudaMemcpyHostToDevice, cs));
    Faces U = {{ux, uy, uz}, {nullptr, nullptr, nullptr}};
    int N = (int)n;
    k_apply_walls<<<grid_for(n_faces(nx, ny, nz)), 256, 0, cs>>>(c, nx, ny, nz, U);
    k_setup_rhs<<<rgrid(N), 256, 0, cs>>>(c, U, nullptr, abs_tol, rel_tol, max_iters);
    enqueue_vcycle(&s, cs, true);
    int st_status = ST_RUNNING;
    for (int it = 0; it <= max_iters + 8; it++) {
        CK(cudaMemcpyAsync(&st_status, &c.st->status, sizeof(int), cudaMemcpyDeviceToHost, cs));
        CK(cudaStreamSynchronize(cs));
        if (st_status != ST_RUNNING) break;
        enqueue_iteration(&s, cs);
    }
    k_grad_p<<<grid_for(n_faces(nx, ny, nz)), 256, 0, cs>>>(c, nx, ny, nz, U);
    CK(cudaPeekAtLastError());
    SolveState fin;
    CK(cudaMemcpyAsync(&fin, c.st, sizeof(fin), cudaMemcpyDeviceToHost, cs));
    CK(cudaStreamSynchronize(cs));
    if (iters) *iters = fin.it;
    if (rTr) *rTr = fin.rTr;
    if (status) *status = fin.status == ST_CONVERGED ? EDGE_OK : (fin.status == ST_NAN ? EDGE_ENAN : EDGE_ENOCONV);
    return EDGE_OK;
}
