// MGPCG pressure projection (sim/mgpcg.py, sim/mgpcg_solid.py) for sm_100a.
//
// One solve is a CUDA graph: set-up kernels, then a conditional WHILE node
// whose body is one CG iteration, then the pressure-gradient update.  The CG
// scalars (alpha, beta, r.r, z.r, the recentering mean) live in device memory
// and are produced by "last block" reductions (per-block float64 partials
// summed in block order, so results are run-to-run deterministic); the body's
// last kernel sets the loop condition, so a solve makes no host round trip.
//
// Layout in HBM.  Every level's r and z, and the fine level's x and p, are
// stored red-black split: cell (i,j,k) of colour c = (i+j+k)&1 lives in plane
// c at slot (i*n1 + j)*H + (k>>1), H = (n2+1)/2.  The six neighbours of a
// colour-c cell at slot e are the other plane's slots e +- n1*H, e +- H,
// e + (k&1) (k+1) and e - 1 + (k&1) (k-1).  A half sweep of colour c therefore
// reads one plane of r and the other plane of z and writes one plane of z, all
// with unit stride, and never touches the half of the grid it does not need.
// The pressure matrix is never stored: A p is recomputed from p where needed.
//
// The all-Neumann recentering (mgpcg.py:169-175) is kept as a pending scalar
// `mean` that every reader of r[0] subtracts and that the r update folds into
// the stored residual.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <set>
#include <tuple>
#include <vector>

#include "edge_common.cuh"

using namespace edge;

namespace {

enum { ST_RUNNING = 0, ST_CONVERGED = 1, ST_NOCONV = 2, ST_NAN = 3 };

struct SolveState {
    double zTr, pAp, rTr, rsum, tol, abs_tol, rel_tol, div_sum;
    float alpha, beta, mean, zsc;
    float zinv;   // 1 / zsc
    int zscaled;  // FP16 level storage: zsc follows the residual's RMS (set_zscale)
    int restart;  // 1: the next z.r epilogue restarts the recursion (beta = 0)
    int pad2;
    int it, max_iters, status, setup;
    int pcur, all_neumann, n_fluid, x_valid;
    unsigned int counter[8];
    unsigned long long kernels;  // kernels of this solver run so far (launch accounting)
};

constexpr size_t kCoarseSmem = 160 * 1024;  // shared memory for the coarse group

// x / d for 0 <= x < 2^31 with one multiply-high (Granlund & Montgomery,
// "Division by invariant integers using multiplication", PLDI 1994, unsigned
// case: l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1,
// q = (mulhi(x, m) + x) >> l; the sum cannot wrap for x < 2^31).
struct FDiv {
    unsigned m;
    int s;
};
inline FDiv make_fdiv(unsigned d) {
    int l = 0;
    while ((1ull << l) < d) l++;
    unsigned long long m = ((1ull << 32) * ((1ull << l) - d)) / d + 1;
    return FDiv{(unsigned)m, l};
}
EDGE_D int fdiv(int x, FDiv f) { return (int)((__umulhi((unsigned)x, f.m) + (unsigned)x) >> f.s); }

// Per-cell neighbour code of the solid solver: which of the six neighbours
// enter the neighbour sum (in range and fluid), whether the cell is fluid,
// and num_fluid_neighbors in bits 8-11 (mgpcg_solid.py:99-130).
enum { NB_XP = 1, NB_XM = 2, NB_YP = 4, NB_YM = 8, NB_ZP = 16, NB_ZM = 32, CELL_FLUID = 64 };

struct Lvl {
    int n0, n1, n2, H;
    int P;               // slots per colour plane, n0*n1*H
    FDiv dH, d1, d2;     // division by H, n1, n2 (index decomposition)
    FDiv dQ;             // division by H/4 (four-slot kernels)
    int vec;             // H % 4 == 0: the level runs the four-slot (float4) kernels
    float* r[2];         // residual planes
    float* z[2];         // preconditioned residual planes
    float* zt;           // third z plane for the fused half-sweep pairs (or NULL)
    unsigned short* code[2];  // solid solver: neighbour codes per plane (else NULL)
    int* bm;             // solid solver: lexicographic mask (level 0: the caller's)
};

struct G {  // what every solver kernel needs
    SolveState* st;
    double* partials;
    cudaGraphConditionalHandle cond;
    int use_cond;  // 0: kernels run outside a graph (eager mode), no loop condition
    cudaGraphConditionalHandle vcond;  // the CG loop body's "still running" IF node
    int use_vcond;
    int nochk;     // 1: launched inside that IF node, the loop is known to be running
    int bt[6];
    int walls;     // bit b set when bt[b] == 2 (device code tests bits: a pointer
                   // into or a run-time index of a kernel-parameter array makes
                   // the compiler copy the parameter struct to local memory)
};

// x[i] of a two-entry parameter array with only constant indices
template <class T>
EDGE_D T pick(const T (&a)[2], int i) { return i ? a[1] : a[0]; }
template <class T>
EDGE_D T pick2(const T (&a)[2][2], int i, int j) {
    return i ? (j ? a[1][1] : a[1][0]) : (j ? a[0][1] : a[0][0]);
}
template <class T>
EDGE_D T pick3(const T (&a)[3], int i) { return i == 0 ? a[0] : (i == 1 ? a[1] : a[2]); }
EDGE_D bool wall(int walls, int side) { return (walls >> side) & 1; }

struct Fine {  // fine-level CG vectors
    float* x[2];
    float* p[2][2];  // [ping-pong buffer][plane]
    float* div;      // lexicographic divergence (edge_mgpcg_get, solid correction)
};

struct Levels {  // the pyramid, for the shared-memory coarse group
    Lvl lv[16];
    int L, lc;
};

struct Ctx {
    Levels lv;
    G g;
    Fine f;
    int csmem;  // dynamic shared memory of k_coarse (bytes)
    int ztype;  // storage of the V-cycle's level arrays: 0 FP32, 1 BF16, 2 FP16 (mixed-precision solvers)
};

EDGE_D void set_cond(const G& g, unsigned v) {
    if (g.use_cond) cudaGraphSetConditional(g.cond, v);
}

EDGE_D bool running(const G& g) { return *((volatile int*)&g.st->status) == ST_RUNNING; }

// In the graph-captured CG loop the V-cycle sits in an IF node whose
// condition the iteration's CG kernels set (k_cg_ap4 clears it, k_cg_xr4
// sets it while the loop runs), so its kernels skip the status load, an L2
// round trip at the head of every launch; launched outside that node they
// read the status and return once the loop has finished.
EDGE_D bool stopped(const G& g) { return !g.nochk && !running(g); }

EDGE_D void set_vcond(const G& g, unsigned v) {
    if (g.use_vcond) cudaGraphSetConditional(g.vcond, v);
}

// every solver kernel counts itself once (block 0, thread 0), including the
// ones that return early once the loop has finished
// Programmatic dependent launch: the CG-loop kernels are launched with
// cudaLaunchAttributeProgrammaticStreamSerialization, so the next kernel's
// launch and block scheduling overlap this one's tail; each of them waits
// here for the previous kernel to complete (and its writes to be visible)
// before reading anything, and lets the next one be scheduled right away.
EDGE_D void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

EDGE_D void count_launch(SolveState* st) {
    if (blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0) atomicAdd(&st->kernels, 1ull);
}

// slot t of a colour plane -> (i, j, kk)
struct Slot {
    int i, j, kk;
};
template <class LV>
EDGE_D Slot slot_of(const LV& L, int t) {
    int row = fdiv(t, L.dH);
    int i = fdiv(row, L.d1);
    return Slot{i, row - i * L.n1, t - row * L.H};
}

// num_fluid_neighbors of the plain solver (mgpcg.py:100-110)
template <class LV>
EDGE_D float nf_walls(int walls, const LV& L, int i, int j, int k) {
    float num = 6.0f;
    if (i <= 0 && wall(walls, 0)) num -= 1.0f;
    if (i >= L.n0 - 1 && wall(walls, 1)) num -= 1.0f;
    if (j <= 0 && wall(walls, 2)) num -= 1.0f;
    if (j >= L.n1 - 1 && wall(walls, 3)) num -= 1.0f;
    if (k <= 0 && wall(walls, 4)) num -= 1.0f;
    if (k >= L.n2 - 1 && wall(walls, 5)) num -= 1.0f;
    return num;
}

// the plain solver's code: every in-range neighbour, every cell fluid
template <class LV>
EDGE_D unsigned range_code(const LV& L, int i, int j, int k) {
    return (i < L.n0 - 1 ? NB_XP : 0) | (i > 0 ? NB_XM : 0) | (j < L.n1 - 1 ? NB_YP : 0) | (j > 0 ? NB_YM : 0) |
           (k < L.n2 - 1 ? NB_ZP : 0) | (k > 0 ? NB_ZM : 0) | CELL_FLUID;
}

template <bool SOLID, class LV>
EDGE_D float nf_of(int walls, const LV& L, unsigned code, int i, int j, int k) {
    return SOLID ? (float)(code >> 8) : nf_walls(walls, L, i, j, k);
}

// neighbour_sum (mgpcg.py:86-99, mgpcg_solid.py:99-111) in the reference's
// order (+x, -x, +y, -y, +z, -z) over the other plane; val(slot, direction)
template <class LV, class F>
EDGE_D float nbr_sum(const LV& L, unsigned code, int e, int k, F val) {
    const int sx = L.n1 * L.H;
    float ret = 0.0f;
    if (code & NB_XP) ret += val(e + sx, 0);
    if (code & NB_XM) ret += val(e - sx, 1);
    if (code & NB_YP) ret += val(e + L.H, 2);
    if (code & NB_YM) ret += val(e - L.H, 3);
    if (code & NB_ZP) ret += val(e + (k & 1), 4);
    if (code & NB_ZM) ret += val(e - 1 + (k & 1), 5);
    return ret;
}

EDGE_D void dir_offset(int d, int& di, int& dj, int& dk) {
    di = d == 0 ? 1 : (d == 1 ? -1 : 0);
    dj = d == 2 ? 1 : (d == 3 ? -1 : 0);
    dk = d == 4 ? 1 : (d == 5 ? -1 : 0);
}

// z of the coarse level at the parent of fine cell (i, j, k) (prolongate,
// mgpcg.py:155-158: z[l][I] += z[l+1][I // 2])
template <class LV>
EDGE_D float parent_z(const LV& C, const float* zc0, const float* zc1, int i, int j, int k) {
    int I = i >> 1, J = j >> 1, K = k >> 1;
    int e = (I * C.n1 + J) * C.H + (K >> 1);
    return ((I + J + K) & 1) ? zc1[e] : zc0[e];
}

// Storage of the V-cycle's level arrays: FP32, or BF16 in the mixed-precision
// solver (the arithmetic stays FP32).  Level 0's r is the CG residual and is
// FP32 in both; pointers are carried as float* and reinterpreted.
template <class ZT>
struct Zs;
template <>
struct Zs<float> {
    static EDGE_D float ld(const float* b, int e) { return __ldg(b + e); }
    static EDGE_D void st(float* b, int e, float v) { b[e] = v; }
    static EDGE_D void ld4(const float* b, int e, float (&v)[4]) {
        float4 t = __ldg(reinterpret_cast<const float4*>(b + e));
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    }
    static EDGE_D void st4(float* b, int e, const float (&v)[4]) {
        *reinterpret_cast<float4*>(b + e) = make_float4(v[0], v[1], v[2], v[3]);
    }
    static EDGE_D void st2(float* b, int e, float x, float y) { *reinterpret_cast<float2*>(b + e) = make_float2(x, y); }
    static EDGE_D float2 ld2(const float* b, int e) { return __ldg(reinterpret_cast<const float2*>(b + e)); }
};
template <>
struct Zs<__nv_bfloat16> {
    static EDGE_D const __nv_bfloat16* h(const float* b) { return reinterpret_cast<const __nv_bfloat16*>(b); }
    static EDGE_D __nv_bfloat16* h(float* b) { return reinterpret_cast<__nv_bfloat16*>(b); }
    static EDGE_D float ld(const float* b, int e) { return __bfloat162float(h(b)[e]); }
    static EDGE_D void st(float* b, int e, float v) { h(b)[e] = __float2bfloat16_rn(v); }
    static EDGE_D void ld4(const float* b, int e, float (&v)[4]) {
        const uint2 u = *reinterpret_cast<const uint2*>(h(b) + e);
        const __nv_bfloat162 a = *reinterpret_cast<const __nv_bfloat162*>(&u.x);
        const __nv_bfloat162 c = *reinterpret_cast<const __nv_bfloat162*>(&u.y);
        v[0] = __low2float(a); v[1] = __high2float(a); v[2] = __low2float(c); v[3] = __high2float(c);
    }
    static EDGE_D void st4(float* b, int e, const float (&v)[4]) {
        __nv_bfloat162 a = __floats2bfloat162_rn(v[0], v[1]), c = __floats2bfloat162_rn(v[2], v[3]);
        uint2 u;
        u.x = *reinterpret_cast<unsigned*>(&a);
        u.y = *reinterpret_cast<unsigned*>(&c);
        *reinterpret_cast<uint2*>(h(b) + e) = u;
    }
    static EDGE_D void st2(float* b, int e, float x, float y) {
        *reinterpret_cast<__nv_bfloat162*>(h(b) + e) = __floats2bfloat162_rn(x, y);
    }
    static EDGE_D float2 ld2(const float* b, int e) {
        const __nv_bfloat162 v = *reinterpret_cast<const __nv_bfloat162*>(h(b) + e);
        return make_float2(__low2float(v), __high2float(v));
    }
};
template <>
struct Zs<__half> {
    static EDGE_D const __half* h(const float* b) { return reinterpret_cast<const __half*>(b); }
    static EDGE_D __half* h(float* b) { return reinterpret_cast<__half*>(b); }
    static EDGE_D float ld(const float* b, int e) { return __half2float(h(b)[e]); }
    static EDGE_D void st(float* b, int e, float v) { h(b)[e] = __float2half_rn(v); }
    static EDGE_D void ld4(const float* b, int e, float (&v)[4]) {
        const uint2 u = *reinterpret_cast<const uint2*>(h(b) + e);
        const __half2 a = *reinterpret_cast<const __half2*>(&u.x);
        const __half2 c = *reinterpret_cast<const __half2*>(&u.y);
        v[0] = __low2float(a); v[1] = __high2float(a); v[2] = __low2float(c); v[3] = __high2float(c);
    }
    static EDGE_D void st4(float* b, int e, const float (&v)[4]) {
        __half2 a = __floats2half2_rn(v[0], v[1]), c = __floats2half2_rn(v[2], v[3]);
        uint2 u;
        u.x = *reinterpret_cast<unsigned*>(&a);
        u.y = *reinterpret_cast<unsigned*>(&c);
        *reinterpret_cast<uint2*>(h(b) + e) = u;
    }
    static EDGE_D void st2(float* b, int e, float x, float y) {
        *reinterpret_cast<__half2*>(h(b) + e) = __floats2half2_rn(x, y);
    }
    static EDGE_D float2 ld2(const float* b, int e) {
        const __half2 v = *reinterpret_cast<const __half2*>(h(b) + e);
        return make_float2(__low2float(v), __high2float(v));
    }
};
// r of a level: FP32 at level 0, else the level storage type
template <class ZT>
EDGE_D float rld(const float* b, int e, int level0) { return level0 ? __ldg(b + e) : Zs<ZT>::ld(b, e); }

// Loads of data that another thread block of the same cluster wrote earlier
// in the same launch: through L2 (ld.global.cg), never the read-only path.
template <class ZT>
struct Zc;
template <>
struct Zc<float> {
    static EDGE_D float ld(const float* b, int e) { return __ldcg(b + e); }
    static EDGE_D float2 ld2(const float* b, int e) { return __ldcg(reinterpret_cast<const float2*>(b + e)); }
    static EDGE_D void ld4(const float* b, int e, float (&v)[4]) {
        float4 t = __ldcg(reinterpret_cast<const float4*>(b + e));
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    }
};
template <>
struct Zc<__nv_bfloat16> {
    static EDGE_D float ld(const float* b, int e) {
        unsigned short u = __ldcg(reinterpret_cast<const unsigned short*>(b) + e);
        return __bfloat162float(__ushort_as_bfloat16(u));
    }
    static EDGE_D float2 ld2(const float* b, int e) {
        unsigned u = __ldcg(reinterpret_cast<const unsigned*>(reinterpret_cast<const unsigned short*>(b) + e));
        const __nv_bfloat162 v = *reinterpret_cast<const __nv_bfloat162*>(&u);
        return make_float2(__low2float(v), __high2float(v));
    }
    static EDGE_D void ld4(const float* b, int e, float (&v)[4]) {
        const uint2 u = __ldcg(reinterpret_cast<const uint2*>(reinterpret_cast<const __nv_bfloat16*>(b) + e));
        const __nv_bfloat162 a = *reinterpret_cast<const __nv_bfloat162*>(&u.x);
        const __nv_bfloat162 c = *reinterpret_cast<const __nv_bfloat162*>(&u.y);
        v[0] = __low2float(a); v[1] = __high2float(a); v[2] = __low2float(c); v[3] = __high2float(c);
    }
};
template <>
struct Zc<__half> {
    static EDGE_D float ld(const float* b, int e) {
        unsigned short u = __ldcg(reinterpret_cast<const unsigned short*>(b) + e);
        return __half2float(__ushort_as_half(u));
    }
    static EDGE_D float2 ld2(const float* b, int e) {
        unsigned u = __ldcg(reinterpret_cast<const unsigned*>(reinterpret_cast<const unsigned short*>(b) + e));
        const __half2 v = *reinterpret_cast<const __half2*>(&u);
        return make_float2(__low2float(v), __high2float(v));
    }
    static EDGE_D void ld4(const float* b, int e, float (&v)[4]) {
        const uint2 u = __ldcg(reinterpret_cast<const uint2*>(reinterpret_cast<const __half*>(b) + e));
        const __half2 a = *reinterpret_cast<const __half2*>(&u.x);
        const __half2 c = *reinterpret_cast<const __half2*>(&u.y);
        v[0] = __low2float(a); v[1] = __high2float(a); v[2] = __low2float(c); v[3] = __high2float(c);
    }
};
template <class ZT>
EDGE_D void rld4(const float* b, int e, int level0, float (&v)[4]) {
    if (level0) Zs<float>::ld4(b, e, v);
    else Zs<ZT>::ld4(b, e, v);
}

// z of the coarse level (global storage) at the parent of fine cell (i, j, k)
template <class ZT, class LV>
EDGE_D float parent_zg(const LV& C, int i, int j, int k) {
    int I = i >> 1, J = j >> 1, K = k >> 1;
    int e = (I * C.n1 + J) * C.H + (K >> 1);
    return Zs<ZT>::ld(pick(C.z, (I + J + K) & 1), e);
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
EDGE_D bool last_block(const G& g, int slot, double (&v)[N]) {
    __shared__ bool am_last;
    block_sum<N>(v);
    int nblk = gridDim.x;
    int b = blockIdx.x;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < N; q++) g.partials[q * nblk + b] = v[q];
        __threadfence();
        unsigned t = atomicAdd(&g.st->counter[slot], 1u);
        am_last = (t == (unsigned)nblk - 1);
    }
    __syncthreads();
    return am_last;
}

// Sum the published partials (fixed order: deterministic) in the last block.
template <int N>
EDGE_D void final_sum(const G& g, int slot, double (&out)[N]) {
    __threadfence();
    int nblk = gridDim.x;
    double v[N];
#pragma unroll
    for (int q = 0; q < N; q++) {
        double s = 0.0;
        for (int b = threadIdx.x; b < nblk; b += blockDim.x) s += __ldcg(g.partials + q * nblk + b);
        v[q] = s;
    }
    block_sum<N>(v);
#pragma unroll
    for (int q = 0; q < N; q++) out[q] = v[q];
    if (threadIdx.x == 0) g.st->counter[slot] = 0;
}

// end of a preconditioner application: z.r, beta, iteration bookkeeping and
// the loop condition (mgpcg.py:221-226, 263-277); thread 0 only
EDGE_D void zr_epilogue(const G& g, double zr) {
    SolveState* st = g.st;
    const double zi = (double)st->zinv;  // z and r of the V-cycle carry the scale zsc each
    double zTr = (double)(float)(zr * zi * zi);
    if (st->setup) {
        st->setup = 0;
        st->zTr = zTr;
        st->beta = 0.0f;
        st->tol = fmax(st->abs_tol, zTr * st->rel_tol);
        if (st->max_iters <= 0) st->status = ST_NOCONV;
    } else {
        st->beta = st->restart ? 0.0f : (float)(zTr / (st->zTr + 1e-12));
        st->restart = 0;
        st->zTr = zTr;
        st->it += 1;
        if (st->it >= st->max_iters) st->status = ST_NOCONV;
    }
    set_cond(g, st->status == ST_RUNNING ? 1u : 0u);
}

// FP16 level storage: the V-cycle runs on the level-0 residual times a power
// of two zsc that brings its RMS near 1 (FP16 keeps 10 bits of mantissa but
// only 5 of exponent); every product and quotient by zsc or zinv is exact, so
// the FP32 and BF16 solvers, whose zsc stays 1, are unaffected.  rr = sum of
// r^2 over n cells.
EDGE_D void set_zscale(SolveState* st, double rr, double n) {
    if (!st->zscaled) return;
    const double rms = sqrt(rr / n);
    int e = 0;
    if (rms > 0.0 && rms < 1e300) e = max(-120, min(120, -(int)lround(log2(rms))));
    st->zsc = ldexpf(1.0f, e);
    st->zinv = ldexpf(1.0f, -e);
}

#define GRID_STRIDE(t, n) for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < (n); t += gridDim.x * blockDim.x)

// ---------------------------------------------------------------------------
// set-up: apply_bc, divergence, solid correction, recentering mean
// ---------------------------------------------------------------------------
struct Faces {
    float* u[3];
    float* f[3];
};

// mgpcg.py:374-392 apply_bc (walls): the wall faces only, one boundary plane
// per blockIdx.y (side = 2 * axis + high)
__global__ void k_apply_walls(G g, int nx, int ny, int nz, Faces U) {
    count_launch(g.st);
    const int side = blockIdx.y;
    if (!wall(g.walls, side)) return;
    const int a = side >> 1, hi = side & 1;
    const int d1 = a == 0 ? ny : nx;  // the plane's two axes, in order
    const int d2 = a == 2 ? ny : nz;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < d1 * d2; t += gridDim.x * blockDim.x) {
        const int u = t / d2, w = t - (t / d2) * d2;
        int e;
        if (a == 0) e = idx3(hi ? nx : 0, u, w, ny, nz);
        else if (a == 1) e = idx3(u, hi ? ny : 0, w, ny + 1, nz);
        else e = idx3(u, w, hi ? nz : 0, ny, nz + 1);
        pick3(U.u, a)[e] = 0.0f;
    }
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
// One thread per slot handles the cell pair k = 2kk (plane (i+j)&1) and
// k = 2kk+1 (the other plane).  x and p need no initialisation: the first
// iteration writes them without reading them.
template <bool SOLID>
__global__ void __launch_bounds__(256) k_setup_rhs(G g, Lvl L, Fine f, Faces U, const float* rhs, double abs_tol,
                                                   double rel_tol, int max_iters) {
    count_launch(g.st);
    const int ny = L.n1, nz = L.n2;
    double v[4] = {0.0, 0.0, 0.0, 0.0};  // sum div (fluid), fluid count, sum r, sum r^2
    GRID_STRIDE(t, L.P) {
        Slot s = slot_of(L, t);
        const int c0 = (s.i + s.j) & 1;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int k = 2 * s.kk + h;
            if (k >= nz) break;
            const int e = idx3(s.i, s.j, k, ny, nz);
            const bool fl = !SOLID || L.bm[e] <= 0;
            float d;
            if (rhs) {
                d = -rhs[e];
            } else if (fl) {
                const int i = s.i, j = s.j;
                float vl = U.u[0][idx3(i, j, k, ny, nz)], vr = U.u[0][idx3(i + 1, j, k, ny, nz)];
                float vb = U.u[1][idx3(i, j, k, ny + 1, nz)], vt = U.u[1][idx3(i, j + 1, k, ny + 1, nz)];
                float va = U.u[2][idx3(i, j, k, ny, nz + 1)], vc = U.u[2][idx3(i, j, k + 1, ny, nz + 1)];
                d = vr - vl + vt - vb + vc - va;
            } else {
                d = 0.0f;
            }
            f.div[e] = d;
            float r = d * -1.0f;
            pick(L.r, c0 ^ h)[t] = r;
            if (fl) {
                v[0] += d;
                v[1] += 1.0;
            }
            v[2] += r;
            v[3] += (double)r * (double)r;
        }
    }
    if (last_block<4>(g, 0, v)) {
        double s[4];
        final_sum<4>(g, 0, s);
        if (threadIdx.x == 0) {
            SolveState* st = g.st;
            st->div_sum = (double)(float)s[0];
            st->n_fluid = (int)s[1];
            st->rsum = s[2];
            st->abs_tol = abs_tol;
            st->rel_tol = rel_tol;
            st->max_iters = max_iters;
            st->it = 0;
            st->status = ST_RUNNING;
            st->setup = 1;
            st->restart = 0;
            st->beta = 0.0f;
            st->alpha = 0.0f;
            st->pcur = 0;
            st->x_valid = 0;
            st->mean = st->all_neumann ? (float)(s[2] / ((double)L.n0 * L.n1 * L.n2)) : 0.0f;
            set_zscale(st, s[3], (double)L.n0 * L.n1 * L.n2);
        }
    }
}

// mgpcg_solid.py:374-383, 422-424: if the fluid divergence sums to > 0,
// subtract its mean from every fluid cell; then the recentering mean.
__global__ void __launch_bounds__(256) k_solid_fix(G g, Lvl L, Fine f) {
    count_launch(g.st);
    SolveState* st = g.st;
    float dsum = (float)st->div_sum;
    bool fix = dsum > 0.0f && st->n_fluid > 0;
    float avg = fix ? dsum / (float)st->n_fluid : 0.0f;
    double v[1] = {0.0};
    GRID_STRIDE(t, L.P) {
        Slot s = slot_of(L, t);
        const int c0 = (s.i + s.j) & 1;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int k = 2 * s.kk + h;
            if (k >= L.n2) break;
            const int e = idx3(s.i, s.j, k, L.n1, L.n2);
            float r = pick(L.r, c0 ^ h)[t];
            if (fix && L.bm[e] <= 0) {
                float d = f.div[e] - avg;
                f.div[e] = d;
                r = d * -1.0f;
                pick(L.r, c0 ^ h)[t] = r;
            }
            v[0] += r;
        }
    }
    if (last_block<1>(g, 1, v)) {
        double s[1];
        final_sum<1>(g, 1, s);
        if (threadIdx.x == 0) st->mean = st->all_neumann ? (float)(s[0] / ((double)L.n0 * L.n1 * L.n2)) : 0.0f;
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

// neighbour codes of one level from its mask: the neighbour_sum conditions
// (mgpcg_solid.py:99-111) and num_fluid_neighbors (mgpcg_solid.py:113-130)
__global__ void __launch_bounds__(256) k_codes(G g, Lvl L) {
    count_launch(g.st);
    const int n1 = L.n1, n2 = L.n2;
    GRID_STRIDE(t, L.n0 * L.n1 * L.n2) {
        int row = fdiv(t, L.d2);
        int k = t - row * n2;
        int i = fdiv(row, L.d1);
        int j = row - i * n1;
        auto solid = [&](int a, int b, int c) { return L.bm[idx3(a, b, c, n1, n2)] > 0; };
        unsigned code = solid(i, j, k) ? 0u : (unsigned)CELL_FLUID;
        int num = 6;
        int I[3] = {i, j, k}, D[3] = {L.n0, n1, n2};
#pragma unroll
        for (int a = 0; a < 3; a++) {
            int up[3] = {i, j, k}, dn[3] = {i, j, k};
            up[a] += 1;
            dn[a] -= 1;
            bool has_up = I[a] < D[a] - 1, has_dn = I[a] > 0;
            bool up_solid = has_up && solid(up[0], up[1], up[2]);
            bool dn_solid = has_dn && solid(dn[0], dn[1], dn[2]);
            if (has_up && !up_solid) code |= 1u << (2 * a);
            if (has_dn && !dn_solid) code |= 2u << (2 * a);
            if (!has_dn && wall(g.walls, 2 * a)) num -= 1;
            else if (dn_solid) num -= 1;
            if (!has_up && wall(g.walls, 2 * a + 1)) num -= 1;
            else if (up_solid) num -= 1;
        }
        code |= (unsigned)num << 8;
        pick(L.code, (i + j + k) & 1)[(i * n1 + j) * L.H + (k >> 1)] = (unsigned short)code;
    }
}

template <bool SOLID>
EDGE_D unsigned code_at(const Lvl& L, int plane, int e, int i, int j, int k) {
    return SOLID ? (unsigned)pick(L.code, plane)[e] : range_code(L, i, j, k);
}

// ---------------------------------------------------------------------------
// CG vector kernels (one thread per slot: the cell pair k = 2kk, 2kk+1)
// ---------------------------------------------------------------------------
// update_p (mgpcg.py:143-145) fused into compute_Ap (mgpcg.py:112-117):
// p_new = z + beta p_old on the fly (also at the stencil neighbours), A p_new
// and the p.Ap partials; the last block forms alpha (mgpcg.py:237-240).
// Products are rounded before the sums (no fused multiply-add), as the
// reference's separate kernels round them.
template <bool SOLID, class ZT>
__global__ void __launch_bounds__(256) k_cg_ap(G g, Lvl L, Fine f) {
    pdl_enter();
    count_launch(g.st);
    // The loop stops unless the iteration's last kernel completes its
    // reduction and asks to continue: a lost reduction can never spin.
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        set_cond(g, 0);
        set_vcond(g, 0);
        if (g.st->it > g.st->max_iters + 8) g.st->status = ST_NOCONV;  // hard cap
    }
    if (!running(g)) return;
    SolveState* st = g.st;
    const int pc = st->pcur;
    const bool first = st->it == 0;  // p = 0 before the first update_p (mgpcg.py:61-66)
    const float beta = st->beta, zinv = st->zinv;
    double v[1] = {0.0};
    GRID_STRIDE(t, L.P) {
        Slot s = slot_of(L, t);
        const int c0 = (s.i + s.j) & 1;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int k = 2 * s.kk + h, pl = c0 ^ h;
            if (k >= L.n2) break;
            const unsigned code = code_at<SOLID>(L, pl, t, s.i, s.j, k);
            float pe = 0.0f;
            if (code & CELL_FLUID) {
                const float* __restrict__ zo = pick(L.z, pl ^ 1);
                const float* __restrict__ po = pick2(f.p, pc, pl ^ 1);
                const float zt = Zs<ZT>::ld(pick(L.z, pl), t) * zinv;
                pe = first ? zt : __fadd_rn(zt, __fmul_rn(beta, __ldg(pick2(f.p, pc, pl) + t)));
                float ns = nbr_sum(L, code, t, k, [&](int e, int) {
                    const float ze = Zs<ZT>::ld(zo, e) * zinv;
                    return first ? ze : __fadd_rn(ze, __fmul_rn(beta, __ldg(po + e)));
                });
                float ape = __fsub_rn(__fmul_rn(nf_of<SOLID>(g.walls, L, code, s.i, s.j, k), pe), ns);
                v[0] += (double)pe * (double)ape;
            }
            pick2(f.p, pc ^ 1, pl)[t] = pe;
        }
    }
    if (last_block<1>(g, 2, v)) {
        double sm[1];
        final_sum<1>(g, 2, sm);
        if (threadIdx.x == 0) {
            double pAp = (double)(float)sm[0];
            st->pAp = pAp;
            st->alpha = (float)(st->zTr / (pAp + 1e-12));
            st->pcur = pc ^ 1;
        }
    }
}

// update_x / update_r (mgpcg.py:133-141) with A p recomputed from p, r.r
// (mgpcg.py:247-249), the convergence test (mgpcg.py:254) and the
// recentering sum (mgpcg.py:169-175).  Solid cells only take the recentering
// (mgpcg_solid.py:197-202).
template <bool SOLID>
__global__ void __launch_bounds__(256) k_cg_xr(G g, Lvl L, Fine f) {
    pdl_enter();
    count_launch(g.st);
    if (!running(g)) return;
    SolveState* st = g.st;
    const float alpha = st->alpha, mean = st->mean;
    const bool first = st->it == 0;  // x = 0 before the first update_x
    const int pc = st->pcur;
    double v[2] = {0.0, 0.0};
    GRID_STRIDE(t, L.P) {
        Slot s = slot_of(L, t);
        const int c0 = (s.i + s.j) & 1;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int k = 2 * s.kk + h, pl = c0 ^ h;
            if (k >= L.n2) break;
            const unsigned code = code_at<SOLID>(L, pl, t, s.i, s.j, k);
            float r = pick(L.r, pl)[t] - mean;
            float* xp = pick(f.x, pl) + t;
            if (code & CELL_FLUID) {
                const float* __restrict__ po = pick2(f.p, pc, pl ^ 1);
                const float pe = __ldg(pick2(f.p, pc, pl) + t);
                *xp = first ? __fmul_rn(alpha, pe) : __fadd_rn(*xp, __fmul_rn(alpha, pe));
                float ns = nbr_sum(L, code, t, k, [&](int e, int) { return __ldg(po + e); });
                float ape = __fsub_rn(__fmul_rn(nf_of<SOLID>(g.walls, L, code, s.i, s.j, k), pe), ns);
                r = __fsub_rn(r, __fmul_rn(alpha, ape));
                v[0] += (double)r * (double)r;
            } else if (first) {
                *xp = 0.0f;
            }
            pick(L.r, pl)[t] = r;
            v[1] += r;
        }
    }
    if (last_block<2>(g, 3, v)) {
        double s[2];
        final_sum<2>(g, 3, s);
        if (threadIdx.x == 0) {
            double rTr = (double)(float)s[0];
            st->rTr = rTr;
            st->rsum = s[1];
            st->x_valid = 1;
            st->mean = st->all_neumann ? (float)(s[1] / ((double)L.n0 * L.n1 * L.n2)) : 0.0f;
            set_zscale(st, rTr, (double)L.n0 * L.n1 * L.n2);
            if (!(rTr == rTr) || rTr > 1e300) st->status = ST_NAN;
            else if (rTr < st->tol) st->status = ST_CONVERGED;
            set_vcond(g, st->status == ST_RUNNING ? 1u : 0u);
        }
    }
}

// ---------------------------------------------------------------------------
// V-cycle (mgpcg.py:177-195)
// ---------------------------------------------------------------------------
// Red-black Gauss-Seidel (mgpcg.py:160-167) runs as half sweeps: a half sweep
// of colour c updates the colour-c cells and reads only cells of the other
// colour, so no update depends on another in the same launch, and a cell's
// own old value is never read.  Hence:
//   * z = 0 before the first down sweep needs no fill: that half sweep reads
//     nothing (HS_FIRST); below the fine level the restriction writes it;
//   * the prolongation z[l] += z[l+1][I/2] (mgpcg.py:155-158) that precedes
//     the up sweeps is applied on the fly to the neighbours the first up half
//     sweep reads (HS_PROLONG): every cell is overwritten by a half sweep
//     before its own value is read again, and solid cells are never read.
enum { HS_FIRST = 0, HS_PLAIN = 1, HS_PROLONG = 2, HS_ZR = 3 };

template <int MODE, bool SOLID, class ZT>
__global__ void __launch_bounds__(256) k_hsweep(G g, Lvl L, Lvl C, int level0, int color) {
    pdl_enter();
    count_launch(g.st);
    if (stopped(g)) {
        if (MODE == HS_ZR && blockIdx.x == 0 && threadIdx.x == 0) set_cond(g, 0);
        return;
    }
    const float mean = level0 ? g.st->mean : 0.0f, zsc = level0 ? g.st->zsc : 1.0f;
    const int oc = color ^ 1;
    const float* __restrict__ rs = pick(L.r, color);
    const float* __restrict__ zo = pick(L.z, oc);
    float* __restrict__ zs = pick(L.z, color);
    double v[1] = {0.0};
    GRID_STRIDE(t, L.P) {
        Slot s = slot_of(L, t);
        const int k = 2 * s.kk + ((s.i + s.j + color) & 1);
        if (k < L.n2) {
            const unsigned code = code_at<SOLID>(L, color, t, s.i, s.j, k);
            if (code & CELL_FLUID) {
                const float rv = (rld<ZT>(rs, t, level0) - mean) * zsc;
                float ns = 0.0f;
                if (MODE == HS_PROLONG) {
                    ns = nbr_sum(L, code, t, k, [&](int e, int d) {
                        int di, dj, dk;
                        dir_offset(d, di, dj, dk);
                        return Zs<ZT>::ld(zo, e) + parent_zg<ZT>(C, s.i + di, s.j + dj, k + dk);
                    });
                } else if (MODE != HS_FIRST) {
                    ns = nbr_sum(L, code, t, k, [&](int e, int) { return Zs<ZT>::ld(zo, e); });
                }
                const float zn = (rv + ns) / nf_of<SOLID>(g.walls, L, code, s.i, s.j, k);
                Zs<ZT>::st(zs, t, zn);
                if (MODE == HS_ZR) v[0] += (double)zn * (double)rv;
            }
        }
        if (MODE == HS_ZR) {
            // the other cell of the slot (final from the previous half sweep)
            const int ko = 2 * s.kk + ((s.i + s.j + oc) & 1);
            if (ko < L.n2 && (code_at<SOLID>(L, oc, t, s.i, s.j, ko) & CELL_FLUID))
                v[0] += (double)Zs<ZT>::ld(zo, t) * (double)((rld<ZT>(pick(L.r, oc), t, level0) - mean) * zsc);
        }
    }
    if (MODE == HS_ZR) {
        // mgpcg.py:263-275: z.r, beta, update bookkeeping, loop condition
        if (last_block<1>(g, 4, v)) {
            double sm[1];
            final_sum<1>(g, 4, sm);
            if (threadIdx.x == 0) zr_epilogue(g, sm[0]);
        }
    }
}

// restrict (mgpcg.py:147-153): r[l+1] = sum over the 8 children of
// (r - A z) / (dim - 1), solid children skipped (mgpcg_solid.py:168-174).
// One thread per coarse cell; the children of (I,J,K) all sit at slot
// (i*n1 + j)*H + K of their planes.  With `first` it also applies the first
// half sweep of the coarse level (z = r / n_fluid on colour 0).
template <bool SOLID, class ZT>
__global__ void __launch_bounds__(256) k_restrict(G g, Lvl F, Lvl C, int level0, int first) {
    pdl_enter();
    count_launch(g.st);
    if (stopped(g)) return;
    const float mean = level0 ? g.st->mean : 0.0f, zsc = level0 ? g.st->zsc : 1.0f;
    GRID_STRIDE(t, C.n0 * C.n1 * C.n2) {
        const int rowc = fdiv(t, C.d2);
        const int K = t - rowc * C.n2;
        const int I = fdiv(rowc, C.d1);
        const int J = rowc - I * C.n1;
        float acc = 0.0f;
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
            for (int b = 0; b < 2; b++)
#pragma unroll
                for (int q = 0; q < 2; q++) {
                    const int i = 2 * I + a, j = 2 * J + b, k = 2 * K + q;
                    const int pl = (i + j + k) & 1;
                    const int e = (i * F.n1 + j) * F.H + K;
                    const unsigned code = code_at<SOLID>(F, pl, e, i, j, k);
                    if (!(code & CELL_FLUID)) continue;
                    const float* __restrict__ zo = pick(F.z, pl ^ 1);
                    float ns = nbr_sum(F, code, e, k, [&](int ee, int) { return Zs<ZT>::ld(zo, ee); });
                    float az = __fsub_rn(__fmul_rn(nf_of<SOLID>(g.walls, F, code, i, j, k), Zs<ZT>::ld(pick(F.z, pl), e)), ns);
                    float res = (rld<ZT>(pick(F.r, pl), e, level0) - mean) * zsc - az;
                    acc += res * 0.5f;
                }
        const int pc = (I + J + K) & 1;
        const int ec = (I * C.n1 + J) * C.H + (K >> 1);
        Zs<ZT>::st(pick(C.r, pc), ec, acc);
        if (first && pc == 0) {
            const unsigned cc = code_at<SOLID>(C, 0, ec, I, J, K);
            if (cc & CELL_FLUID) Zs<ZT>::st(C.z[0], ec, (acc + 0.0f) / nf_of<SOLID>(g.walls, C, cc, I, J, K));
        }
    }
}

// ---------------------------------------------------------------------------
// Four slots per thread (levels with H % 4 == 0): one float4 per plane row
// segment instead of four scalar loads, same arithmetic in the same order.
// ---------------------------------------------------------------------------
EDGE_D void ld4(const float* p, float (&v)[4]) {
    float4 t = __ldg(reinterpret_cast<const float4*>(p));
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
}
// coherent load (the thread itself rewrites these words in the same kernel)
EDGE_D void ld4c(const float* p, float (&v)[4]) {
    float4 t = *reinterpret_cast<const float4*>(p);
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
}
EDGE_D void st4(float* p, const float (&v)[4]) { *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]); }

// slots kk0..kk0+3 of row (i, j); t0 = the first slot's index in a plane
struct Quad {
    int i, j, kk0, t0;
};
// p ? b : a for p in {0, 1} on the bits, so that the choice between two
// array elements at constant indices is not turned back into one load at a
// run-time index (which puts the array in local memory)
EDGE_D float bsel(int p, float a, float b) {
    const unsigned mask = 0u - (unsigned)p;
    return __uint_as_float((__float_as_uint(a) & ~mask) | (__float_as_uint(b) & mask));
}

template <class LV>
EDGE_D Quad quad_of(const LV& L, int t) {
    int row = fdiv(t, L.dQ);
    int i = fdiv(row, L.d1);
    int kk0 = (t - row * (L.H >> 2)) << 2;
    return Quad{i, row - i * L.n1, kk0, row * L.H + kk0};
}

// codes of the four cells of plane `plane` (parity p: k = 2 kk + p)
template <bool SOLID>
EDGE_D void quad_codes(const Lvl& L, int plane, const Quad& q, int p, unsigned (&code)[4]) {
    if (SOLID) {
        ushort4 c = *reinterpret_cast<const ushort4*>(pick(L.code, plane) + q.t0);
        code[0] = c.x; code[1] = c.y; code[2] = c.z; code[3] = c.w;
    } else {
#pragma unroll
        for (int m = 0; m < 4; m++) code[m] = range_code(L, q.i, q.j, 2 * (q.kk0 + m) + p);
    }
}

// neighbour sums of the four cells over the other plane, in the reference's
// order; v4(slot, out[4]) loads four consecutive other-plane values, v1(slot)
// one.  With PRO each neighbour also takes pz(i, j, k), the coarse level's z
// at its parent (the prolongation, added before the neighbour enters the sum).
template <bool PRO, class LV, class V4, class V1, class PZ>
EDGE_D void quad_nbr_sum(const LV& L, const Quad& q, int p, const unsigned (&code)[4], V4 v4, V1 v1, PZ pz,
                         float (&ns)[4]) {
    const int sx = L.n1 * L.H;
    float xp[4] = {0, 0, 0, 0}, xm[4] = {0, 0, 0, 0}, yp[4] = {0, 0, 0, 0}, ym[4] = {0, 0, 0, 0};
    float ov[4], o[6];
    if (q.i < L.n0 - 1) v4(q.t0 + sx, xp);
    if (q.i > 0) v4(q.t0 - sx, xm);
    if (q.j < L.n1 - 1) v4(q.t0 + L.H, yp);
    if (q.j > 0) v4(q.t0 - L.H, ym);
    v4(q.t0, ov);
    o[0] = (p == 0 && q.kk0 > 0) ? v1(q.t0 - 1) : 0.0f;  // slot kk0-1
    o[1] = ov[0]; o[2] = ov[1]; o[3] = ov[2]; o[4] = ov[3];
    o[5] = (p == 1 && q.kk0 + 4 < L.H) ? v1(q.t0 + 4) : 0.0f;  // slot kk0+4
#pragma unroll
    for (int m = 0; m < 4; m++) {
        const unsigned c = code[m];
        const int k = 2 * (q.kk0 + m) + p;
        float vxp = xp[m], vxm = xm[m], vyp = yp[m], vym = ym[m], vzp = bsel(p, o[m + 1], o[m + 2]),
              vzm = bsel(p, o[m], o[m + 1]);
        if (PRO) {
            if (c & NB_XP) vxp = vxp + pz(q.i + 1, q.j, k);
            if (c & NB_XM) vxm = vxm + pz(q.i - 1, q.j, k);
            if (c & NB_YP) vyp = vyp + pz(q.i, q.j + 1, k);
            if (c & NB_YM) vym = vym + pz(q.i, q.j - 1, k);
            if (c & NB_ZP) vzp = vzp + pz(q.i, q.j, k + 1);
            if (c & NB_ZM) vzm = vzm + pz(q.i, q.j, k - 1);
        }
        float r = 0.0f;
        if (c & NB_XP) r += vxp;
        if (c & NB_XM) r += vxm;
        if (c & NB_YP) r += vyp;
        if (c & NB_YM) r += vym;
        if (c & NB_ZP) r += vzp;
        if (c & NB_ZM) r += vzm;
        ns[m] = r;
    }
}

struct NoParent {
    EDGE_D float operator()(int, int, int) const { return 0.0f; }
};

// The prolongation terms a quad's six neighbour directions take
// (prolongate, mgpcg.py:155-158: the coarse z at each neighbour's parent),
// gathered with vector loads: when the fine row length is a multiple of 8,
// the parents of cells k = 2 (kk0 + m) + p, m = 0..3, are coarse cells
// K = kk0 + m of at most three coarse columns, two consecutive slots of each
// colour plane per column.  ld2(plane, slot) returns slots slot, slot + 1 of
// a coarse plane, ld1(plane, slot) one.  Values of neighbours outside the grid
// are 0 and never used.
struct QParents {
    float xp[4], xm[4], yp[4], ym[4], zp[4], zm[4];
};
template <class LV, class CV, class L2, class L1>
EDGE_D void quad_parents(const LV& F, const CV& C, int i, int j, int kk0, int p, L2 ld2, L1 ld1, QParents& o) {
    const int I = i >> 1, J = j >> 1, s = kk0 >> 1;
    auto col = [&](int Ic, int Jc, float(&v)[4]) {
        const int base = (Ic * C.n1 + Jc) * C.H + s;
        const int A = (Ic + Jc) & 1;
        const float2 a = ld2(A, base), b = ld2(A ^ 1, base);
        v[0] = a.x; v[1] = b.x; v[2] = a.y; v[3] = b.y;
    };
    float c[4];
    col(I, J, c);
#pragma unroll
    for (int m = 0; m < 4; m++) { o.xp[m] = o.xm[m] = o.yp[m] = o.ym[m] = c[m]; }
    // the x and y neighbours on the side of the other parent
    if (i & 1) {
        if (i + 1 < F.n0) col(I + 1, J, o.xp);
    } else if (i > 0) {
        col(I - 1, J, o.xm);
    }
    if (j & 1) {
        if (j + 1 < F.n1) col(I, J + 1, o.yp);
    } else if (j > 0) {
        col(I, J - 1, o.ym);
    }
    // z: parents of k + 1 and k - 1 are K = kk0 + m + p and kk0 + m + p - 1
    const int A = (I + J) & 1;
    const int rowb = (I * C.n1 + J) * C.H;
    const float lo = (p == 0 && kk0 > 0) ? ld1(A ^ 1, rowb + s - 1) : 0.0f;            // K = kk0 - 1
    const float hi = (p == 1 && 2 * kk0 + 8 < F.n2) ? ld1(A, rowb + s + 2) : 0.0f;    // K = kk0 + 4
    const float e6[6] = {lo, c[0], c[1], c[2], c[3], hi};                               // K = kk0 - 1 .. kk0 + 4
#pragma unroll
    for (int m = 0; m < 4; m++) {
        o.zp[m] = bsel(p, e6[m + 1], e6[m + 2]);
        o.zm[m] = bsel(p, e6[m], e6[m + 1]);
    }
}

// quad_nbr_sum with the prolongation terms of quad_parents
template <class LV, class V4, class V1>
EDGE_D void quad_nbr_sum_pro(const LV& L, const Quad& q, int p, const unsigned (&code)[4], V4 v4, V1 v1,
                             const QParents& P, float (&ns)[4]) {
    const int sx = L.n1 * L.H;
    float xp[4] = {0, 0, 0, 0}, xm[4] = {0, 0, 0, 0}, yp[4] = {0, 0, 0, 0}, ym[4] = {0, 0, 0, 0};
    float ov[4], o[6];
    if (q.i < L.n0 - 1) v4(q.t0 + sx, xp);
    if (q.i > 0) v4(q.t0 - sx, xm);
    if (q.j < L.n1 - 1) v4(q.t0 + L.H, yp);
    if (q.j > 0) v4(q.t0 - L.H, ym);
    v4(q.t0, ov);
    o[0] = (p == 0 && q.kk0 > 0) ? v1(q.t0 - 1) : 0.0f;
    o[1] = ov[0]; o[2] = ov[1]; o[3] = ov[2]; o[4] = ov[3];
    o[5] = (p == 1 && q.kk0 + 4 < L.H) ? v1(q.t0 + 4) : 0.0f;
#pragma unroll
    for (int m = 0; m < 4; m++) {
        const unsigned c = code[m];
        float vxp = xp[m], vxm = xm[m], vyp = yp[m], vym = ym[m], vzp = bsel(p, o[m + 1], o[m + 2]),
              vzm = bsel(p, o[m], o[m + 1]);
        if (c & NB_XP) vxp = vxp + P.xp[m];
        if (c & NB_XM) vxm = vxm + P.xm[m];
        if (c & NB_YP) vyp = vyp + P.yp[m];
        if (c & NB_YM) vym = vym + P.ym[m];
        if (c & NB_ZP) vzp = vzp + P.zp[m];
        if (c & NB_ZM) vzm = vzm + P.zm[m];
        float r = 0.0f;
        if (c & NB_XP) r += vxp;
        if (c & NB_XM) r += vxm;
        if (c & NB_YP) r += vyp;
        if (c & NB_YM) r += vym;
        if (c & NB_ZP) r += vzp;
        if (c & NB_ZM) r += vzm;
        ns[m] = r;
    }
}

// The coarse levels lc..L-1 of a V-cycle in one thread block out of shared
// memory (same red-black layout): down sweeps + restriction, 20 bottom
// sweeps, prolongation + up sweeps (mgpcg.py:177-195); z[lc] is written back
// for the prolongation into level lc-1.  Levels of at most 32 slots per plane
// run on one warp.  With ZR (the whole grid fits, lc == 0) it also forms z.r
// and runs the end-of-iteration bookkeeping.
struct CLvl {
    int n0, n1, n2, H, P;
    FDiv dH, d1, d2, dQ;
    int vec;
    int roff, zoff, coff;  // float offsets of the r and z planes, ushort offset of the codes
};

// The level structs of a launch's Levels parameter, copied to shared memory
// with constant indices (a run-time index into the parameter would put the
// whole parameter in local memory).
EDGE_D void copy_levels(const Levels& a, Lvl* sl) {
#pragma unroll
    for (int l = 0; l < 16; l++)
        if ((int)threadIdx.x == l && l < a.L) sl[l] = a.lv[l];
}

// Body of the coarse group (levels lc..L-1, lvs in shared memory), run by one
// thread block; COH: r[lc] was written earlier in the same launch by another
// thread block of the cluster (coherent loads).
template <bool ZR, bool SOLID, class ZT, bool COH>
EDGE_D void coarse_body(const G& g, const Lvl* lvs, int L, int lc, float* sh, CLvl* cl) {
    if (threadIdx.x == 0) {
        // per level: r plane 0, r plane 1, z plane 0, z plane 1 (floats); the
        // solid codes (two planes per level) follow all the floats
        int off = 0;
        for (int l = lc; l < L; l++) {
            const Lvl& V = lvs[l];
            CLvl q;
            q.n0 = V.n0; q.n1 = V.n1; q.n2 = V.n2; q.H = V.H; q.P = V.P;
            q.dH = V.dH; q.d1 = V.d1; q.d2 = V.d2; q.dQ = V.dQ;
            q.vec = V.vec;
            q.roff = off;
            q.zoff = off + 2 * V.P;
            off += 4 * V.P;
            cl[l] = q;
        }
        int coff = 2 * off;  // in unsigned shorts from the start of shared memory
        for (int l = lc; l < L; l++) {
            cl[l].coff = coff;
            coff += 2 * cl[l].P;
        }
    }
    __syncthreads();
    unsigned short* codes = reinterpret_cast<unsigned short*>(sh);
    const float mean = lc == 0 ? g.st->mean : 0.0f, zsc = lc == 0 ? g.st->zsc : 1.0f;
    {
        // kLoadBatch loads in flight per thread before their shared-memory
        // stores (one at a time, each would wait for the L2 round trip)
        constexpr int kLoadBatch = 8;
        const CLvl& q = cl[lc];
        for (int e0 = threadIdx.x; e0 < 2 * q.P; e0 += kLoadBatch * blockDim.x) {
            float v[kLoadBatch];
#pragma unroll
            for (int u = 0; u < kLoadBatch; u++) {
                const int e = e0 + u * blockDim.x;
                v[u] = 0.0f;
                if (e < 2 * q.P) {
                    const float* src = e < q.P ? lvs[lc].r[0] : lvs[lc].r[1];
                    const int ee = e < q.P ? e : e - q.P;
                    v[u] = ((COH ? Zc<ZT>::ld(src, ee) : rld<ZT>(src, ee, lc == 0)) - mean) * zsc;
                }
            }
#pragma unroll
            for (int u = 0; u < kLoadBatch; u++)
                if (e0 + u * blockDim.x < 2 * q.P) sh[q.roff + e0 + u * blockDim.x] = v[u];
        }
        if (SOLID)
            for (int l = lc; l < L; l++) {
                const CLvl& u = cl[l];
                for (int e = threadIdx.x; e < 2 * u.P; e += blockDim.x)
                    codes[u.coff + e] = e < u.P ? lvs[l].code[0][e] : lvs[l].code[1][e - u.P];
            }
    }
    __syncthreads();
    // one half sweep; mode 0: from zero, 1: plain, 2: with the prolongation of
    // l+1.  Levels of at most 64 slots per plane run on warp 0 alone; levels
    // with H % 4 == 0 take four slots per thread (float4 shared-memory loads;
    // plane offsets are multiples of four floats).
    auto half = [&](int l, int color, int mode) {
        const CLvl& q = cl[l];
        const bool small = q.P <= 64;
        if (!small || threadIdx.x < 32) {
            const int step = small ? 32 : blockDim.x;
            const float* r = sh + q.roff + color * q.P;
            float* z = sh + q.zoff + color * q.P;
            const float* zo = sh + q.zoff + (color ^ 1) * q.P;
            const unsigned short* cd = codes + q.coff + color * q.P;
            const CLvl& u = cl[mode == 2 ? l + 1 : l];
            const float* zc0 = sh + u.zoff;
            const float* zc1 = zc0 + u.P;
            auto pz = [&](int i, int j, int k) { return parent_z(u, zc0, zc1, i, j, k); };
            if (q.vec) {
                const int nq = q.P >> 2;
                for (int t = threadIdx.x; t < nq; t += step) {
                    const Quad qd = quad_of(q, t);
                    const int p = (qd.i + qd.j + color) & 1;
                    unsigned code[4];
                    if (SOLID) {
                        ushort4 c4 = *reinterpret_cast<const ushort4*>(cd + qd.t0);
                        code[0] = c4.x; code[1] = c4.y; code[2] = c4.z; code[3] = c4.w;
                    } else {
#pragma unroll
                        for (int m = 0; m < 4; m++) code[m] = range_code(q, qd.i, qd.j, 2 * (qd.kk0 + m) + p);
                    }
                    float ns[4] = {0.0f, 0.0f, 0.0f, 0.0f};
                    auto v4 = [&](int e, float(&o)[4]) {
                        float4 w = *reinterpret_cast<const float4*>(zo + e);
                        o[0] = w.x; o[1] = w.y; o[2] = w.z; o[3] = w.w;
                    };
                    auto v1 = [&](int e) { return zo[e]; };
                    if (mode == 1) {
                        quad_nbr_sum<false>(q, qd, p, code, v4, v1, NoParent(), ns);
                    } else if (mode == 2 && q.n2 % 8 == 0) {
                        QParents P;
                        quad_parents(
                            q, u, qd.i, qd.j, qd.kk0, p,
                            [&](int pl, int e) { return *reinterpret_cast<const float2*>((pl ? zc1 : zc0) + e); },
                            [&](int pl, int e) { return (pl ? zc1 : zc0)[e]; }, P);
                        quad_nbr_sum_pro(q, qd, p, code, v4, v1, P, ns);
                    } else if (mode == 2) {
                        quad_nbr_sum<true>(q, qd, p, code, v4, v1, pz, ns);
                    }
                    float4 rv = *reinterpret_cast<const float4*>(r + qd.t0);
                    float4 zv = *reinterpret_cast<const float4*>(z + qd.t0);
                    float rr[4] = {rv.x, rv.y, rv.z, rv.w}, zz[4] = {zv.x, zv.y, zv.z, zv.w};
#pragma unroll
                    for (int m = 0; m < 4; m++)
                        if (code[m] & CELL_FLUID)
                            zz[m] = (rr[m] + ns[m]) / nf_of<SOLID>(g.walls, q, code[m], qd.i, qd.j, 2 * (qd.kk0 + m) + p);
                    *reinterpret_cast<float4*>(z + qd.t0) = make_float4(zz[0], zz[1], zz[2], zz[3]);
                }
            } else {
                for (int t = threadIdx.x; t < q.P; t += step) {
                    Slot s = slot_of(q, t);
                    const int k = 2 * s.kk + ((s.i + s.j + color) & 1);
                    if (k >= q.n2) continue;
                    const unsigned code = SOLID ? (unsigned)cd[t] : range_code(q, s.i, s.j, k);
                    if (!(code & CELL_FLUID)) continue;
                    float ns = 0.0f;
                    if (mode == 1) {
                        ns = nbr_sum(q, code, t, k, [&](int e, int) { return zo[e]; });
                    } else if (mode == 2) {
                        ns = nbr_sum(q, code, t, k, [&](int e, int d) {
                            int di, dj, dk;
                            dir_offset(d, di, dj, dk);
                            return zo[e] + pz(s.i + di, s.j + dj, k + dk);
                        });
                    }
                    z[t] = (r[t] + ns) / nf_of<SOLID>(g.walls, q, code, s.i, s.j, k);
                }
            }
        }
        if (small) __syncwarp();
        else __syncthreads();
    };
    // down
    for (int l = lc; l < L - 1; l++) {
        half(l, 0, 0);
        half(l, 1, 1);
        half(l, 0, 1);
        half(l, 1, 1);
        __syncthreads();
        // restrict into r[l+1]
        const CLvl& q = cl[l];
        const CLvl& u = cl[l + 1];
        const int m = u.n0 * u.n1 * u.n2;
        for (int ce = threadIdx.x; ce < m; ce += blockDim.x) {
            const int rowc = fdiv(ce, u.d2);
            const int K = ce - rowc * u.n2;
            const int I = fdiv(rowc, u.d1);
            const int J = rowc - I * u.n1;
            float acc = 0.0f;
            for (int aa = 0; aa < 2; aa++)
                for (int b = 0; b < 2; b++)
                    for (int cc = 0; cc < 2; cc++) {
                        const int i = 2 * I + aa, j = 2 * J + b, k = 2 * K + cc;
                        const int pl = (i + j + k) & 1;
                        const int e = (i * q.n1 + j) * q.H + K;
                        const unsigned code =
                            SOLID ? (unsigned)codes[q.coff + pl * q.P + e] : range_code(q, i, j, k);
                        if (!(code & CELL_FLUID)) continue;
                        const float* zo = sh + q.zoff + (pl ^ 1) * q.P;
                        float ns = nbr_sum(q, code, e, k, [&](int ee, int) { return zo[ee]; });
                        float az = __fsub_rn(__fmul_rn(nf_of<SOLID>(g.walls, q, code, i, j, k), sh[q.zoff + pl * q.P + e]),
                                             ns);
                        float res = sh[q.roff + pl * q.P + e] - az;
                        acc += res * 0.5f;
                    }
            sh[u.roff + ((I + J + K) & 1) * u.P + (I * u.n1 + J) * u.H + (K >> 1)] = acc;
        }
        __syncthreads();
    }
    // bottom (mgpcg.py:186-189): 20 red-black iterations.  When the level
    // has at most blockDim.x slots per plane, thread t owns slot t of both
    // planes with its codes, divisors, residuals and neighbour offsets held in
    // registers for all 40 half sweeps, and only the warps that own slots
    // synchronise (named barrier 1); the arithmetic is half()'s.
    if (cl[L - 1].P <= (int)blockDim.x) {
        const CLvl& q = cl[L - 1];
        const int nt = (q.P + 31) & ~31;
        const int t = threadIdx.x;
        if (t < nt) {
            bool act[2];
            unsigned code[2];
            float nf[2], rr[2];
            int kk[2];
            const int sx = q.n1 * q.H;
            Slot s = slot_of(q, t < q.P ? t : 0);
#pragma unroll
            for (int c = 0; c < 2; c++) {
                kk[c] = 2 * s.kk + ((s.i + s.j + c) & 1);
                act[c] = t < q.P && kk[c] < q.n2;
                code[c] = 0;
                nf[c] = 1.0f;
                rr[c] = 0.0f;
                if (act[c]) {
                    code[c] = SOLID ? (unsigned)codes[q.coff + c * q.P + t] : range_code(q, s.i, s.j, kk[c]);
                    act[c] = (code[c] & CELL_FLUID) != 0;
                    nf[c] = nf_of<SOLID>(g.walls, q, code[c], s.i, s.j, kk[c]);
                    rr[c] = sh[q.roff + c * q.P + t];
                }
            }
            float* z0 = sh + q.zoff;
            float* z1 = z0 + q.P;
            auto sweep = [&](int c, bool from_zero) {
                if (act[c]) {
                    const float* zo = c ? z0 : z1;
                    float ns = 0.0f;
                    if (!from_zero) {
                        const int k = kk[c];
                        if (code[c] & NB_XP) ns += zo[t + sx];
                        if (code[c] & NB_XM) ns += zo[t - sx];
                        if (code[c] & NB_YP) ns += zo[t + q.H];
                        if (code[c] & NB_YM) ns += zo[t - q.H];
                        if (code[c] & NB_ZP) ns += zo[t + (k & 1)];
                        if (code[c] & NB_ZM) ns += zo[t - 1 + (k & 1)];
                    }
                    (c ? z1 : z0)[t] = (rr[c] + ns) / nf[c];
                }
                asm volatile("bar.sync 1, %0;" ::"r"(nt) : "memory");
            };
            sweep(0, true);
            sweep(1, false);
            for (int it = 1; it < 20; it++) {
                sweep(0, false);
                sweep(1, false);
            }
        }
    } else {
        half(L - 1, 0, 0);
        half(L - 1, 1, 1);
        for (int it = 1; it < 20; it++) {
            half(L - 1, 0, 1);
            half(L - 1, 1, 1);
        }
    }
    __syncthreads();
    // up
    for (int l = L - 2; l >= lc; l--) {
        half(l, 1, 2);
        half(l, 0, 1);
        half(l, 1, 1);
        half(l, 0, 1);
        __syncthreads();
    }
    // write back z[lc] (solid cells keep their last value, never read)
    {
        const CLvl& q = cl[lc];
        for (int e = threadIdx.x; e < 2 * q.P; e += blockDim.x) {
            float* dst = e < q.P ? lvs[lc].z[0] : lvs[lc].z[1];
            Zs<ZT>::st(dst, e < q.P ? e : e - q.P, sh[q.zoff + e]);
        }
    }
    if (ZR) {
        const CLvl& q = cl[lc];
        double v[1] = {0.0};
        for (int e = threadIdx.x; e < 2 * q.P; e += blockDim.x) {
            const int color = e < q.P ? 0 : 1, t = e - color * q.P;
            Slot s = slot_of(q, t);
            const int k = 2 * s.kk + ((s.i + s.j + color) & 1);
            if (k >= q.n2) continue;
            const bool fl = SOLID ? (codes[q.coff + e] & CELL_FLUID) != 0 : true;
            if (fl) v[0] += (double)sh[q.zoff + e] * (double)sh[q.roff + e];
        }
        block_sum<1>(v);
        if (threadIdx.x == 0) zr_epilogue(g, v[0]);
    }
}

template <bool ZR, bool SOLID, class ZT>
__global__ void __launch_bounds__(1024) k_coarse(G g, Levels a) {
    pdl_enter();
    extern __shared__ float sh[];
    __shared__ CLvl cl[16];
    __shared__ Lvl sl[16];
    count_launch(g.st);
    if (stopped(g)) {
        if (ZR && threadIdx.x == 0) set_cond(g, 0);
        return;
    }
    copy_levels(a, sl);
    __syncthreads();
    coarse_body<ZR, SOLID, ZT, false>(g, sl, a.L, a.lc, sh, cl);
}

template <int MODE, bool SOLID, class ZT>
__global__ void __launch_bounds__(256) k_hsweep4(G g, Lvl L, Lvl C, int level0, int color) {
    pdl_enter();
    count_launch(g.st);
    if (stopped(g)) {
        if (MODE == HS_ZR && blockIdx.x == 0 && threadIdx.x == 0) set_cond(g, 0);
        return;
    }
    const float mean = level0 ? g.st->mean : 0.0f, zsc = level0 ? g.st->zsc : 1.0f;
    const int oc = color ^ 1;
    const float* __restrict__ rs = pick(L.r, color);
    const float* __restrict__ zo = pick(L.z, oc);
    float* __restrict__ zs = pick(L.z, color);
    double v[1] = {0.0};
    // two slots' loads in flight per thread (the pointers are restrict-qualified,
    // so the second iteration's loads may move above the first one's stores)
#pragma unroll 2
    GRID_STRIDE(t, L.n0 * L.n1 * (L.H >> 2)) {
        const Quad q = quad_of(L, t);
        const int p = (q.i + q.j + color) & 1;
        unsigned code[4];
        quad_codes<SOLID>(L, color, q, p, code);
        float rv[4], ns[4] = {0.0f, 0.0f, 0.0f, 0.0f}, zn[4];
        rld4<ZT>(rs, q.t0, level0, rv);
        if (MODE != HS_FIRST) {
            auto v4 = [&](int e, float(&o)[4]) { Zs<ZT>::ld4(zo, e, o); };
            auto v1 = [&](int e) { return Zs<ZT>::ld(zo, e); };
            if (MODE == HS_PROLONG && L.n2 % 8 == 0) {
                QParents P;
                quad_parents(L, C, q.i, q.j, q.kk0, p, [&](int pl, int e) { return Zs<ZT>::ld2(pick(C.z, pl), e); },
                             [&](int pl, int e) { return Zs<ZT>::ld(pick(C.z, pl), e); }, P);
                quad_nbr_sum_pro(L, q, p, code, v4, v1, P, ns);
            } else if (MODE == HS_PROLONG)
                quad_nbr_sum<true>(L, q, p, code, v4, v1,
                                   [&](int i, int j, int k) { return parent_zg<ZT>(C, i, j, k); }, ns);
            else
                quad_nbr_sum<false>(L, q, p, code, v4, v1, NoParent(), ns);
        }
#pragma unroll
        for (int m = 0; m < 4; m++) {
            rv[m] = (rv[m] - mean) * zsc;
            zn[m] = (code[m] & CELL_FLUID) ? (rv[m] + ns[m]) / nf_of<SOLID>(g.walls, L, code[m], q.i, q.j, 2 * (q.kk0 + m) + p)
                                           : 0.0f;
            if (MODE == HS_ZR && (code[m] & CELL_FLUID)) v[0] += (double)zn[m] * (double)rv[m];
        }
        Zs<ZT>::st4(zs, q.t0, zn);
        if (MODE == HS_ZR) {
            // the other cells of the slots (final from the previous half sweep)
            unsigned co[4];
            quad_codes<SOLID>(L, oc, q, p ^ 1, co);
            float ro[4], zz[4];
            rld4<ZT>(pick(L.r, oc), q.t0, level0, ro);
            Zs<ZT>::ld4(zo, q.t0, zz);
#pragma unroll
            for (int m = 0; m < 4; m++)
                if (co[m] & CELL_FLUID) v[0] += (double)zz[m] * (double)((ro[m] - mean) * zsc);
        }
    }
    if (MODE == HS_ZR) {
        if (last_block<1>(g, 4, v)) {
            double sm[1];
            final_sum<1>(g, 4, sm);
            if (threadIdx.x == 0) zr_epilogue(g, sm[0]);
        }
    }
}

template <bool SOLID, class ZT>
__global__ void __launch_bounds__(256) k_cg_ap4(G g, Lvl L, Fine f) {
    pdl_enter();
    count_launch(g.st);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        set_cond(g, 0);
        set_vcond(g, 0);
        if (g.st->it > g.st->max_iters + 8) g.st->status = ST_NOCONV;  // hard cap
    }
    if (!running(g)) return;
    SolveState* st = g.st;
    const int pc = st->pcur;
    const bool first = st->it == 0;
    const float beta = st->beta, zinv = st->zinv;
    double v[1] = {0.0};
    GRID_STRIDE(t, L.n0 * L.n1 * (L.H >> 2)) {
        const Quad q = quad_of(L, t);
        const int c0 = (q.i + q.j) & 1;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int pl = c0 ^ h;
            unsigned code[4];
            quad_codes<SOLID>(L, pl, q, h, code);
            const float* __restrict__ zo = pick(L.z, pl ^ 1);
            const float* __restrict__ po = pick2(f.p, pc, pl ^ 1);
            auto pn4 = [&](const float* zz, const float* pp, int e, float(&o)[4]) {
                Zs<ZT>::ld4(zz, e, o);
#pragma unroll
                for (int m = 0; m < 4; m++) o[m] = o[m] * zinv;
                if (!first) {
                    float b[4];
                    ld4(pp + e, b);
#pragma unroll
                    for (int m = 0; m < 4; m++) o[m] = __fadd_rn(o[m], __fmul_rn(beta, b[m]));
                }
            };
            float pe[4], ns[4];
            pn4(pick(L.z, pl), pick2(f.p, pc, pl), q.t0, pe);
            quad_nbr_sum<false>(
                L, q, h, code, [&](int e, float(&o)[4]) { pn4(zo, po, e, o); },
                [&](int e) {
                    const float ze = Zs<ZT>::ld(zo, e) * zinv;
                    return first ? ze : __fadd_rn(ze, __fmul_rn(beta, __ldg(po + e)));
                },
                NoParent(), ns);
#pragma unroll
            for (int m = 0; m < 4; m++) {
                if (code[m] & CELL_FLUID) {
                    float nf = nf_of<SOLID>(g.walls, L, code[m], q.i, q.j, 2 * (q.kk0 + m) + h);
                    float ape = __fsub_rn(__fmul_rn(nf, pe[m]), ns[m]);
                    v[0] += (double)pe[m] * (double)ape;
                } else {
                    pe[m] = 0.0f;
                }
            }
            st4(pick2(f.p, pc ^ 1, pl) + q.t0, pe);
        }
    }
    if (last_block<1>(g, 2, v)) {
        double sm[1];
        final_sum<1>(g, 2, sm);
        if (threadIdx.x == 0) {
            double pAp = (double)(float)sm[0];
            st->pAp = pAp;
            st->alpha = (float)(st->zTr / (pAp + 1e-12));
            st->pcur = pc ^ 1;
        }
    }
}

template <bool SOLID>
__global__ void __launch_bounds__(256) k_cg_xr4(G g, Lvl L, Fine f) {
    pdl_enter();
    count_launch(g.st);
    if (!running(g)) return;
    SolveState* st = g.st;
    const float alpha = st->alpha, mean = st->mean;
    const bool first = st->it == 0;
    const int pc = st->pcur;
    double v[2] = {0.0, 0.0};
    GRID_STRIDE(t, L.n0 * L.n1 * (L.H >> 2)) {
        const Quad q = quad_of(L, t);
        const int c0 = (q.i + q.j) & 1;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int pl = c0 ^ h;
            unsigned code[4];
            quad_codes<SOLID>(L, pl, q, h, code);
            const float* __restrict__ po = pick2(f.p, pc, pl ^ 1);
            float pe[4], ns[4], r[4], x[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            ld4(pick2(f.p, pc, pl) + q.t0, pe);
            ld4c(pick(L.r, pl) + q.t0, r);
            if (!first) ld4c(pick(f.x, pl) + q.t0, x);
            quad_nbr_sum<false>(
                L, q, h, code, [&](int e, float(&o)[4]) { ld4(po + e, o); }, [&](int e) { return __ldg(po + e); },
                NoParent(), ns);
#pragma unroll
            for (int m = 0; m < 4; m++) {
                r[m] = r[m] - mean;
                if (code[m] & CELL_FLUID) {
                    x[m] = first ? __fmul_rn(alpha, pe[m]) : __fadd_rn(x[m], __fmul_rn(alpha, pe[m]));
                    float nf = nf_of<SOLID>(g.walls, L, code[m], q.i, q.j, 2 * (q.kk0 + m) + h);
                    float ape = __fsub_rn(__fmul_rn(nf, pe[m]), ns[m]);
                    r[m] = __fsub_rn(r[m], __fmul_rn(alpha, ape));
                    v[0] += (double)r[m] * (double)r[m];
                }
                v[1] += r[m];
            }
            st4(pick(f.x, pl) + q.t0, x);
            st4(pick(L.r, pl) + q.t0, r);
        }
    }
    if (last_block<2>(g, 3, v)) {
        double s[2];
        final_sum<2>(g, 3, s);
        if (threadIdx.x == 0) {
            double rTr = (double)(float)s[0];
            st->rTr = rTr;
            st->rsum = s[1];
            st->x_valid = 1;
            st->mean = st->all_neumann ? (float)(s[1] / ((double)L.n0 * L.n1 * L.n2)) : 0.0f;
            set_zscale(st, rTr, (double)L.n0 * L.n1 * L.n2);
            if (!(rTr == rTr) || rTr > 1e300) st->status = ST_NAN;
            else if (rTr < st->tol) st->status = ST_CONVERGED;
            set_vcond(g, st->status == ST_RUNNING ? 1u : 0u);
        }
    }
}

// ---------------------------------------------------------------------------
// Two consecutive half sweeps in one launch, through a shared-memory tile
// with a halo.  A block owns TI x TJ rows (i, j) of the level, every row
// whole in k.  It stages the other colour's z of its rows plus two on each
// side (with the coarse parent's z added when the first sweep is the
// prolongation sweep), runs the first half sweep (colour cA) on its rows plus
// one on each side - the halo cells are computed by both neighbouring blocks
// from the same inputs, so they agree bit for bit, and only the owner stores
// them - then the second half sweep (colour cB) on its rows, reading the
// first sweep's results from shared memory.  Each cell's arithmetic is
// k_hsweep4's, in the same order (the first sweep's values pass through the
// level's storage type before the second reads them, as they do through
// global memory between two launches).
//
// The second sweep's results go to zBout, a plane other than the one colour
// cB is staged from: another block may still be staging those rows as its
// halo.  The host tracks which of the level's three z planes (z[0], z[1], zt)
// holds each colour after every launch.
// ---------------------------------------------------------------------------
constexpr size_t kPairSmemMax = 200 * 1024;
constexpr int kPairDefault = 0;

// shared memory of a pair launch with TI x TJ owned rows of H slots
inline size_t pair_smem(int TI, int TJ, int H) {
    return (size_t)((TI + 4) * (TJ + 4) + (TI + 2) * (TJ + 2)) * H * sizeof(float);
}

// v rounded to the level's storage type (what a store and a reload return)
template <class ZT>
EDGE_D float zt_round(float v) { return v; }
template <>
EDGE_D float zt_round<__nv_bfloat16>(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }
template <>
EDGE_D float zt_round<__half>(float v) { return __half2float(__float2half_rn(v)); }

// nbr_sum over a staged tile: the same directions, order and code tests;
// W = row width of the staged tile, s = the cell's index in it
template <class F>
EDGE_D float nbr_sum_s(unsigned code, int s, int k, int W, int H, F val) {
    float ret = 0.0f;
    if (code & NB_XP) ret += val(s + W * H);
    if (code & NB_XM) ret += val(s - W * H);
    if (code & NB_YP) ret += val(s + H);
    if (code & NB_YM) ret += val(s - H);
    if (code & NB_ZP) ret += val(s + (k & 1));
    if (code & NB_ZM) ret += val(s - 1 + (k & 1));
    return ret;
}

template <int MA, int MB, bool SOLID, class ZT, int TI, int TJ>
__global__ void __launch_bounds__(256) k_hs_pair(G g, Lvl L, Lvl C, int level0, int cA, float* zBout) {
    pdl_enter();
    count_launch(g.st);
    if (stopped(g)) {
        if (MB == HS_ZR && blockIdx.x == 0 && threadIdx.x == 0) set_cond(g, 0);
        return;
    }
    extern __shared__ float sm[];
    const int H = L.H, cB = cA ^ 1;
    constexpr int WB = TJ + 4, WA = TJ + 2, RB = (TI + 4) * WB, RA = (TI + 2) * WA;
    float* zB = sm;
    float* zA = sm + RB * H;
    const float mean = level0 ? g.st->mean : 0.0f, zsc = level0 ? g.st->zsc : 1.0f;
    const int nti = (L.n0 + TI - 1) / TI, ntj = (L.n1 + TJ - 1) / TJ;
    const float* __restrict__ zo = pick(L.z, cB);
    float* __restrict__ zAg = pick(L.z, cA);
    float* __restrict__ zBg = zBout;
    const float* __restrict__ rA = pick(L.r, cA);
    const float* __restrict__ rB = pick(L.r, cB);
    double v[1] = {0.0};
    for (int tile = blockIdx.x; tile < nti * ntj; tile += gridDim.x) {
        const int i0 = (tile / ntj) * TI, j0 = (tile % ntj) * TJ;
        // 1. colour cB's z on the rows i0-2 .. i0+TI+1, j0-2 .. j0+TJ+1
        if (MA != HS_FIRST) {
            for (int t = threadIdx.x; t < RB * H; t += blockDim.x) {
                const int row = fdiv(t, L.dH), kk = t - row * H;
                const int i = i0 - 2 + row / WB, j = j0 - 2 + row % WB;
                float z = 0.0f;
                if (i >= 0 && i < L.n0 && j >= 0 && j < L.n1) {
                    const int k = 2 * kk + ((i + j + cB) & 1);
                    z = Zs<ZT>::ld(zo, (i * L.n1 + j) * H + kk);
                    if (MA == HS_PROLONG && k < L.n2) z = z + parent_zg<ZT>(C, i, j, k);
                }
                zB[t] = z;
            }
            __syncthreads();
        }
        // 2. first half sweep (colour cA) on the rows i0-1 .. i0+TI, j0-1 .. j0+TJ
        for (int t = threadIdx.x; t < RA * H; t += blockDim.x) {
            const int row = fdiv(t, L.dH), kk = t - row * H;
            const int ii = row / WA, jj = row % WA;
            const int i = i0 - 1 + ii, j = j0 - 1 + jj;
            float zn = 0.0f;
            if (i >= 0 && i < L.n0 && j >= 0 && j < L.n1) {
                const int k = 2 * kk + ((i + j + cA) & 1);
                const int e = (i * L.n1 + j) * H + kk;
                const unsigned code = k < L.n2 ? code_at<SOLID>(L, cA, e, i, j, k) : 0u;
                if (code & CELL_FLUID) {
                    const float rv = (rld<ZT>(rA, e, level0) - mean) * zsc;
                    float ns = 0.0f;
                    if (MA != HS_FIRST)
                        ns = nbr_sum_s(code, ((ii + 1) * WB + (jj + 1)) * H + kk, k, WB, H,
                                       [&](int q) { return zB[q]; });
                    zn = (rv + ns) / nf_of<SOLID>(g.walls, L, code, i, j, k);
                }
                if (ii >= 1 && ii <= TI && jj >= 1 && jj <= TJ) Zs<ZT>::st(zAg, e, zn);
                zn = zt_round<ZT>(zn);
            }
            zA[t] = zn;
        }
        __syncthreads();
        // 3. second half sweep (colour cB) on the owned rows
        for (int t = threadIdx.x; t < TI * TJ * H; t += blockDim.x) {
            const int row = fdiv(t, L.dH), kk = t - row * H;
            const int ii = row / TJ, jj = row % TJ;
            const int i = i0 + ii, j = j0 + jj;
            if (i >= L.n0 || j >= L.n1) continue;
            const int k = 2 * kk + ((i + j + cB) & 1);
            const int e = (i * L.n1 + j) * H + kk;
            const int sa = ((ii + 1) * WA + (jj + 1)) * H + kk;
            const unsigned code = k < L.n2 ? code_at<SOLID>(L, cB, e, i, j, k) : 0u;
            float zn = 0.0f;
            float rv = 0.0f;
            if (code & CELL_FLUID) {
                rv = (rld<ZT>(rB, e, level0) - mean) * zsc;
                const float ns = nbr_sum_s(code, sa, k, WA, H, [&](int q) { return zA[q]; });
                zn = (rv + ns) / nf_of<SOLID>(g.walls, L, code, i, j, k);
                if (MB == HS_ZR) v[0] += (double)zn * (double)rv;
            }
            Zs<ZT>::st(zBg, e, zn);
            if (MB == HS_ZR) {
                // the colour-cA cell of the same slot, final after the first sweep
                const int kA = 2 * kk + ((i + j + cA) & 1);
                if (kA < L.n2 && (code_at<SOLID>(L, cA, e, i, j, kA) & CELL_FLUID))
                    v[0] += (double)zA[sa] * (double)((rld<ZT>(rA, e, level0) - mean) * zsc);
            }
        }
        __syncthreads();  // the tile's shared arrays are refilled by the next tile
    }
    if (MB == HS_ZR) {
        if (last_block<1>(g, 4, v)) {
            double sm1[1];
            final_sum<1>(g, 4, sm1);
            if (threadIdx.x == 0) zr_epilogue(g, sm1[0]);
        }
    }
}

// restriction, four coarse cells (I, J, K0..K0+3) per thread: their children
// are slots K0..K0+3 of both planes in the four fine rows (2I+a, 2J+b)
template <bool SOLID, class ZT>
__global__ void __launch_bounds__(256) k_restrict4(G g, Lvl F, Lvl C, int level0, int first) {
    pdl_enter();
    count_launch(g.st);
    if (stopped(g)) return;
    const float mean = level0 ? g.st->mean : 0.0f, zsc = level0 ? g.st->zsc : 1.0f;
    const int nq = F.H >> 2;  // == C.n2 / 4
    GRID_STRIDE(t, C.n0 * C.n1 * nq) {
        const int rowc = fdiv(t, F.dQ);
        const int K0 = (t - rowc * nq) << 2;
        const int I = fdiv(rowc, C.d1);
        const int J = rowc - I * C.n1;
        float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
            for (int b = 0; b < 2; b++) {
                const int i = 2 * I + a, j = 2 * J + b;
                const Quad q{i, j, K0, (i * F.n1 + j) * F.H + K0};
                const int c0 = (i + j) & 1;
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int pl = c0 ^ h;
                    unsigned code[4];
                    quad_codes<SOLID>(F, pl, q, h, code);
                    const float* __restrict__ zo = pick(F.z, pl ^ 1);
                    float ns[4], zc[4], rc[4];
                    quad_nbr_sum<false>(
                        F, q, h, code, [&](int e, float(&o)[4]) { Zs<ZT>::ld4(zo, e, o); },
                        [&](int e) { return Zs<ZT>::ld(zo, e); }, NoParent(), ns);
                    Zs<ZT>::ld4(pick(F.z, pl), q.t0, zc);
                    rld4<ZT>(pick(F.r, pl), q.t0, level0, rc);
#pragma unroll
                    for (int m = 0; m < 4; m++) {
                        if (!(code[m] & CELL_FLUID)) continue;
                        float nf = nf_of<SOLID>(g.walls, F, code[m], i, j, 2 * (K0 + m) + h);
                        float az = __fsub_rn(__fmul_rn(nf, zc[m]), ns[m]);
                        float res = (rc[m] - mean) * zsc - az;
                        acc[m] += res * 0.5f;
                    }
                }
            }
        // coarse cells K0, K0+2 sit in plane (I+J)&1, K0+1, K0+3 in the other,
        // at slots ecb, ecb+1
        const int ecb = (I * C.n1 + J) * C.H + (K0 >> 1);
        const int pa = (I + J) & 1;
        Zs<ZT>::st2(pick(C.r, pa), ecb, acc[0], acc[2]);
        Zs<ZT>::st2(pick(C.r, pa ^ 1), ecb, acc[1], acc[3]);
        if (first) {
            // first half sweep of the coarse level: z = r / n_fluid on colour 0
            const int m0 = pa;  // the colour-0 cells are m0 and m0 + 2
            float zz[2];
#pragma unroll
            for (int u = 0; u < 2; u++) {
                const int m = m0 + 2 * u, K = K0 + m;
                const unsigned cc = SOLID ? (unsigned)C.code[0][ecb + u] : range_code(C, I, J, K);
                zz[u] = (cc & CELL_FLUID) ? (acc[m] + 0.0f) / nf_of<SOLID>(g.walls, C, cc, I, J, K) : 0.0f;
            }
            Zs<ZT>::st2(C.z[0], ecb, zz[0], zz[1]);
        }
    }
}

// mgpcg.py:406-432 subtract_grad_p (p = x, get_result mgpcg.py:77-85) + the
// wall part of the final apply_bc; Poisson_with_buffer's force (mgpcg.py:448-479).
// One thread per slot: the faces on the low side of its two cells in each
// axis, and the high boundary faces of cells on the high boundary.
EDGE_D void face_update(const G& g, const Faces& U, int a, int e, float gr, bool at_wall) {
    float* ua = pick3(U.u, a);
    float* fa = pick3(U.f, a);
    float u = ua[e] - gr;
    if (at_wall) u = 0.0f;
    ua[e] = u;
    if (fa) fa[e] = -gr;
}

__global__ void __launch_bounds__(256) k_grad_p(G g, Lvl L, Fine f, Faces U) {
    count_launch(g.st);
    const bool xv = g.st->x_valid != 0;  // x = 0 when no iteration ran
    const int nx = L.n0, ny = L.n1, nz = L.n2, sx = L.n1 * L.H;
    GRID_STRIDE(t, L.P) {
        const Slot s = slot_of(L, t);
        const int i = s.i, j = s.j, c0 = (i + j) & 1;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int k = 2 * s.kk + h, pl = c0 ^ h;
            if (k >= nz) break;
            const float* xo = pick(f.x, pl ^ 1);
            const float xc = xv ? pick(f.x, pl)[t] : 0.0f;
            const float xl = (xv && i > 0) ? xo[t - sx] : 0.0f;
            face_update(g, U, 0, idx3(i, j, k, ny, nz), xc - xl, i == 0 && wall(g.walls, 0));
            if (i == nx - 1) face_update(g, U, 0, idx3(nx, j, k, ny, nz), 0.0f - xc, wall(g.walls, 1));
            const float yl = (xv && j > 0) ? xo[t - L.H] : 0.0f;
            face_update(g, U, 1, idx3(i, j, k, ny + 1, nz), xc - yl, j == 0 && wall(g.walls, 2));
            if (j == ny - 1) face_update(g, U, 1, idx3(i, ny, k, ny + 1, nz), 0.0f - xc, wall(g.walls, 3));
            const float zl = (xv && k > 0) ? xo[t - 1 + (k & 1)] : 0.0f;
            face_update(g, U, 2, idx3(i, j, k, ny, nz + 1), xc - zl, k == 0 && wall(g.walls, 4));
            if (k == nz - 1) face_update(g, U, 2, idx3(i, j, nz, ny, nz + 1), 0.0f - xc, wall(g.walls, 5));
        }
    }
}

// red-black planes <-> lexicographic field of one level; `valid` (may be
// NULL) gates the planes' content (x before the first update reads as 0)
__global__ void k_set_restart(SolveState* st) {
    if (threadIdx.x == 0) st->restart = 1;
}

// zsc of an FP16 solver from the RMS of level 0's r planes (V-cycle calls)
__global__ void __launch_bounds__(256) k_zscale(G g, Lvl L) {
    double v[1] = {0.0};
    GRID_STRIDE(t, L.P) {
        const Slot sl = slot_of(L, t);
        const int c0 = (sl.i + sl.j) & 1;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            if (2 * sl.kk + h >= L.n2) break;
            const float r = pick(L.r, c0 ^ h)[t];
            v[0] += (double)r * (double)r;
        }
    }
    if (last_block<1>(g, 5, v)) {
        double sm[1];
        final_sum<1>(g, 5, sm);
        if (threadIdx.x == 0) set_zscale(g.st, sm[0], (double)L.n0 * L.n1 * L.n2);
    }
}

__global__ void k_from_rb(SolveState* st, Lvl L, const float* p0, const float* p1, float* dst, const int* valid,
                          int ztype, const float* scale) {
    if (st) count_launch(st);
    const bool ok = valid == nullptr || *valid != 0;
    GRID_STRIDE(t, L.n0 * L.n1 * L.n2) {
        int row = fdiv(t, L.d2);
        int k = t - row * L.n2;
        int i = fdiv(row, L.d1);
        int j = row - i * L.n1;
        const float* p = ((i + j + k) & 1) ? p1 : p0;
        const int e = row * L.H + (k >> 1);
        const float v = ztype == 1 ? Zs<__nv_bfloat16>::ld(p, e) : (ztype == 2 ? Zs<__half>::ld(p, e) : p[e]);
        dst[t] = ok ? (scale ? v * *scale : v) : 0.0f;
    }
}

__global__ void k_to_rb(Lvl L, const float* src, float* p0, float* p1, int ztype) {
    GRID_STRIDE(t, L.n0 * L.n1 * L.n2) {
        int row = fdiv(t, L.d2);
        int k = t - row * L.n2;
        int i = fdiv(row, L.d1);
        int j = row - i * L.n1;
        float* p = ((i + j + k) & 1) ? p1 : p0;
        const int e = row * L.H + (k >> 1);
        if (ztype == 1) Zs<__nv_bfloat16>::st(p, e, src[t]);
        else if (ztype == 2) Zs<__half>::st(p, e, src[t]);
        else p[e] = src[t];
    }
}

// num_fluid_neighbors from the lexicographic mask (edge_mgpcg_apply_A)
EDGE_D float n_fluid_lex(int walls, const Lvl& L, int i, int j, int k) {
    float num = 6.0f;
    int I[3] = {i, j, k}, D[3] = {L.n0, L.n1, L.n2};
#pragma unroll
    for (int a = 0; a < 3; a++) {
        if (I[a] <= 0 && wall(walls, 2 * a)) num -= 1.0f;
        else if (L.bm && I[a] > 0) {
            int e = idx3(i - (a == 0), j - (a == 1), k - (a == 2), L.n1, L.n2);
            if (__ldg(L.bm + e) > 0) num -= 1.0f;
        }
        if (I[a] >= D[a] - 1 && wall(walls, 2 * a + 1)) num -= 1.0f;
        else if (L.bm && I[a] < D[a] - 1) {
            int e = idx3(i + (a == 0), j + (a == 1), k + (a == 2), L.n1, L.n2);
            if (__ldg(L.bm + e) > 0) num -= 1.0f;
        }
    }
    return num;
}

EDGE_D bool is_fluid(const int* bm, int e) { return bm == nullptr || __ldg(bm + e) <= 0; }

__global__ void k_apply_A(G g, Lvl L, const float* p, float* Ap) {
    int n = L.n0 * L.n1 * L.n2;
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    if (!is_fluid(L.bm, e)) {
        Ap[e] = 0.0f;
        return;
    }
    int k = e % L.n2, j = (e / L.n2) % L.n1, i = e / (L.n1 * L.n2);
    int I[3] = {i, j, k}, D[3] = {L.n0, L.n1, L.n2};
    int stride[3] = {L.n1 * L.n2, L.n2, 1};
    float ns = 0.0f;
    for (int a = 0; a < 3; a++) {
        if (I[a] < D[a] - 1 && is_fluid(L.bm, e + stride[a])) ns += p[e + stride[a]];
        if (I[a] > 0 && is_fluid(L.bm, e - stride[a])) ns += p[e - stride[a]];
    }
    Ap[e] = __fsub_rn(__fmul_rn(n_fluid_lex(g.walls, L, i, j, k), p[e]), ns);
}

// the same operator in float64 (the FP64 reference solve of the precision study)
__global__ void k_apply_A64(G g, Lvl L, const double* p, double* Ap) {
    int n = L.n0 * L.n1 * L.n2;
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    if (!is_fluid(L.bm, e)) {
        Ap[e] = 0.0;
        return;
    }
    int k = e % L.n2, j = (e / L.n2) % L.n1, i = e / (L.n1 * L.n2);
    int I[3] = {i, j, k}, D[3] = {L.n0, L.n1, L.n2};
    int stride[3] = {L.n1 * L.n2, L.n2, 1};
    double ns = 0.0;
    for (int a = 0; a < 3; a++) {
        if (I[a] < D[a] - 1 && is_fluid(L.bm, e + stride[a])) ns += p[e + stride[a]];
        if (I[a] > 0 && is_fluid(L.bm, e - stride[a])) ns += p[e - stride[a]];
    }
    Ap[e] = (double)n_fluid_lex(g.walls, L, i, j, k) * p[e] - ns;
}

// Iterative refinement (mixed-precision solves): r = b - A x with b, x and
// the arithmetic in float64, r stored as the float32 right-hand side of the
// next inner solve, and sums of r^2 and b^2 (fluid cells) into out[0..1]
// (last block, block order); then x += d for the inner solve's correction d.
__global__ void __launch_bounds__(256) k_refine_residual(G g, Lvl L, const double* b, const double* x, float* r32,
                                                         double* out, int slot) {
    const int n = L.n0 * L.n1 * L.n2;
    double v[2] = {0.0, 0.0};
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        double r = 0.0;
        if (is_fluid(L.bm, e)) {
            const int k = e % L.n2, j = (e / L.n2) % L.n1, i = e / (L.n1 * L.n2);
            const int I[3] = {i, j, k}, D[3] = {L.n0, L.n1, L.n2};
            const int stride[3] = {L.n1 * L.n2, L.n2, 1};
            double ns = 0.0;
#pragma unroll
            for (int a = 0; a < 3; a++) {
                if (I[a] < D[a] - 1 && is_fluid(L.bm, e + stride[a])) ns += x[e + stride[a]];
                if (I[a] > 0 && is_fluid(L.bm, e - stride[a])) ns += x[e - stride[a]];
            }
            const double be = b[e];
            r = be - ((double)n_fluid_lex(g.walls, L, i, j, k) * x[e] - ns);
            v[0] += r * r;
            v[1] += be * be;
        }
        r32[e] = (float)r;
    }
    if (last_block<2>(g, slot, v)) {
        double sm[2];
        final_sum<2>(g, slot, sm);
        if (threadIdx.x == 0) {
            out[0] = sm[0];
            out[1] = sm[1];
        }
    }
}

__global__ void k_refine_update(long long n, double* x, const float* d) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        x[e] += (double)d[e];
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

// reduction and sweep kernels loop over their slots with at most this many
// blocks (8 per SM), which bounds the last-block atomics
constexpr int kMaxBlocks = 148 * 8;
inline int rgrid(long long n) { return (int)std::max<long long>(1, std::min<long long>(grid_for(n), kMaxBlocks)); }

// plane length rounded to 64 floats, so every plane starts 256-byte aligned
inline size_t plane_alloc(long long P) { return (size_t)((P + 63) / 64 * 64); }

void set_level_dims(Lvl& V, int n0, int n1, int n2) {
    V.n0 = n0; V.n1 = n1; V.n2 = n2;
    V.H = (n2 + 1) / 2;
    V.P = n0 * n1 * V.H;
    V.dH = make_fdiv((unsigned)V.H);
    V.d1 = make_fdiv((unsigned)n1);
    V.d2 = make_fdiv((unsigned)n2);
    V.vec = V.H % 4 == 0;
    V.dQ = make_fdiv((unsigned)std::max(1, V.H / 4));
}

// A captured solve graph holds every pointer its kernels read or write: the
// face velocities and forces (Poisson), the right-hand side and the solution
// (solve), so all of them key it.
struct GraphKey {
    const void* a[8];
    double abs_tol, rel_tol;
    int max_iters;
    bool operator<(const GraphKey& o) const {
        return std::tie(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], abs_tol, rel_tol, max_iters) <
               std::tie(o.a[0], o.a[1], o.a[2], o.a[3], o.a[4], o.a[5], o.a[6], o.a[7], o.abs_tol, o.rel_tol,
                        o.max_iters);
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
};

int alloc(Solver* s, void** p, size_t bytes) {
    CK(cudaMalloc(p, bytes));
    s->allocs.push_back(*p);
    return EDGE_OK;
}

// The levels lc..L-1 that fit in kCoarseSmem of shared memory together go to
// k_coarse; the finer ones run half-sweep kernels.
void plan_coarse(Ctx& c, bool solid) {
    Levels& V = c.lv;
    for (int lc = 0; lc < V.L; lc++) {
        size_t floats = 0, codes = 0;
        for (int l = lc; l < V.L; l++) {
            floats += 4 * (size_t)V.lv[l].P;
            codes += 2 * (size_t)V.lv[l].P;
        }
        size_t bytes = floats * sizeof(float) + (solid ? codes * sizeof(unsigned short) : 0) + 16;
        if (bytes <= kCoarseSmem || lc == V.L - 1) {
            V.lc = lc;
            c.csmem = (int)bytes;
            return;
        }
    }
}

template <class ZT>
static int coarse_smem_attrs(int bytes) {
    CK(cudaFuncSetAttribute(k_coarse<true, false, ZT>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    CK(cudaFuncSetAttribute(k_coarse<false, false, ZT>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    CK(cudaFuncSetAttribute(k_coarse<true, true, ZT>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    CK(cudaFuncSetAttribute(k_coarse<false, true, ZT>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    return EDGE_OK;
}

template <class ZT>
static int pair_attrs_z();

int prepare_coarse_kernels(const Ctx& c) {
    if ((size_t)c.csmem > kCoarseSmem) return EDGE_EINVAL;  // the coarsest level alone must fit
    if (c.csmem > 48 * 1024) {
        int r = coarse_smem_attrs<float>(c.csmem);
        if (r == EDGE_OK) r = coarse_smem_attrs<__nv_bfloat16>(c.csmem);
        if (r == EDGE_OK) r = coarse_smem_attrs<__half>(c.csmem);
        if (r != EDGE_OK) return r;
    }
    // the fused half-sweep pairs' tiles (up to kPairSmemMax bytes), once per device
    static std::mutex mu;
    static std::set<int> done;
    int dev = 0;
    CK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    if (done.count(dev)) return EDGE_OK;
    int r = pair_attrs_z<float>();
    if (r == EDGE_OK) r = pair_attrs_z<__nv_bfloat16>();
    if (r == EDGE_OK) r = pair_attrs_z<__half>();
    if (r == EDGE_OK) done.insert(dev);
    return r;
}

// Blocks of kernel k (block threads, smem bytes of dynamic shared memory)
// resident on the whole current device at once; cached per (device, kernel,
// shape).  The solver's kernels loop over their slots, so a grid of at most
// this many blocks runs in one wave with no block waiting for a free SM (the
// CG kernels, 3-4 blocks per SM by their registers, measured 10-20% faster
// than with 8 blocks per SM in 2-3 waves).
static int wave_blocks(const void* k, int block, size_t smem) {
    static std::map<std::tuple<int, const void*, int, size_t>, int> cache;
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        (void)cudaGetLastError();
        return kMaxBlocks;
    }
    const auto key = std::make_tuple(dev, k, block, smem);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    int per_sm = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, block, smem) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        (void)cudaGetLastError();
        return kMaxBlocks;
    }
    const int n = std::max(1, per_sm * sms);
    cache[key] = n;
    return n;
}

// launch with the programmatic-dependent-launch attribute (see pdl_enter),
// at most one wave of blocks
template <class... KArgs, class... Args>
static void launch_pdl(void (*k)(KArgs...), int grid, int block, size_t smem, cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(std::min(grid, wave_blocks(reinterpret_cast<const void*>(k), block, smem)));
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k, args...);
}

// Fused half-sweep pairs (k_hs_pair): 0 off, else the tile of rows a block
// owns: 1 = 8 x 4, 2 = 8 x 8, 3 = 16 x 8.  EDGE_MGPCG_PAIR overrides the
// default; read once per process.
static int pair_mode() {
    static const int m = [] {
        const char* e = getenv("EDGE_MGPCG_PAIR");
        const int v = e ? atoi(e) : kPairDefault;
        return v >= 0 && v <= 3 ? v : kPairDefault;
    }();
    return m;
}
static void pair_tile(int mode, int& ti, int& tj) {
    ti = mode == 3 ? 16 : 8;
    tj = mode == 1 ? 4 : 8;
}

// whether level l runs its sweeps as fused pairs
static bool use_pair(const Ctx& c, int l) {
    const Lvl& L = c.lv.lv[l];
    const int m = pair_mode();
    if (m == 0 || L.zt == nullptr || l >= c.lv.lc) return false;
    int ti, tj;
    pair_tile(m, ti, tj);
    return pair_smem(ti, tj, L.H) <= kPairSmemMax;
}

// level L with colour q's z held in plane zq
inline Lvl with_z(const Lvl& L, int q, float* zq) {
    Lvl x = L;
    x.z[q] = zq;
    return x;
}

// Where level l's z is after its up sweeps (what the prolongation into level
// l - 1 reads): a paired level below the fine one ends with colour 1 in zt.
static Lvl up_layout(const Ctx& c, int l) {
    const Lvl& L = c.lv.lv[l];
    return l > 0 && use_pair(c, l) ? with_z(L, 1, L.zt) : L;
}

template <int MA, int MB, bool S, class ZT>
static void launch_pair(const Ctx& c, const Lvl& L, const Lvl& C, int l0, int cA, float* out, cudaStream_t st) {
    int ti, tj;
    const int m = pair_mode();
    pair_tile(m, ti, tj);
    const size_t sm = pair_smem(ti, tj, L.H);
    const int tiles = ((L.n0 + ti - 1) / ti) * ((L.n1 + tj - 1) / tj);
    const int g = std::min(tiles, kMaxBlocks);
    if (m == 1) launch_pdl(k_hs_pair<MA, MB, S, ZT, 8, 4>, g, 256, sm, st, c.g, L, C, l0, cA, out);
    else if (m == 2) launch_pdl(k_hs_pair<MA, MB, S, ZT, 8, 8>, g, 256, sm, st, c.g, L, C, l0, cA, out);
    else launch_pdl(k_hs_pair<MA, MB, S, ZT, 16, 8>, g, 256, sm, st, c.g, L, C, l0, cA, out);
}

template <int MA, int MB, bool S, class ZT>
static int pair_attrs_t() {
    const int b = (int)kPairSmemMax;
    CK(cudaFuncSetAttribute(k_hs_pair<MA, MB, S, ZT, 8, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
    CK(cudaFuncSetAttribute(k_hs_pair<MA, MB, S, ZT, 8, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
    CK(cudaFuncSetAttribute(k_hs_pair<MA, MB, S, ZT, 16, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
    return EDGE_OK;
}
template <bool S, class ZT>
static int pair_attrs_s() {
    int r = pair_attrs_t<HS_FIRST, HS_PLAIN, S, ZT>();
    if (r == EDGE_OK) r = pair_attrs_t<HS_PLAIN, HS_PLAIN, S, ZT>();
    if (r == EDGE_OK) r = pair_attrs_t<HS_PROLONG, HS_PLAIN, S, ZT>();
    if (r == EDGE_OK) r = pair_attrs_t<HS_PLAIN, HS_ZR, S, ZT>();
    return r;
}
template <class ZT>
static int pair_attrs_z() {
    int r = pair_attrs_s<false, ZT>();
    return r == EDGE_OK ? pair_attrs_s<true, ZT>() : r;
}

// one half sweep of colour `color`, unfused
template <int MODE, bool S, class ZT>
static void launch_hs(const Ctx& c, const Lvl& L, const Lvl& C, int l0, int color, cudaStream_t stream) {
    if (L.vec)
        launch_pdl(k_hsweep4<MODE, S, ZT>, rgrid((long long)L.n0 * L.n1 * (L.H / 4)), 256, 0, stream, c.g, L, C, l0,
                   color);
    else
        launch_pdl(k_hsweep<MODE, S, ZT>, rgrid(L.P), 256, 0, stream, c.g, L, C, l0, color);
}

template <bool S, class ZT>
static void launch_restrict(const Ctx& c, const Lvl& L, const Lvl& C, int l0, int first, cudaStream_t stream) {
    if (L.vec)
        launch_pdl(k_restrict4<S, ZT>, rgrid((long long)C.n0 * C.n1 * (L.H / 4)), 256, 0, stream, c.g, L, C, l0, first);
    else
        launch_pdl(k_restrict<S, ZT>, rgrid((long long)C.n0 * C.n1 * C.n2), 256, 0, stream, c.g, L, C, l0, first);
}

// the descent of a V-cycle: levels 0..lc-1 (sweeps and restrictions).
// Sweeps per level (mgpcg.py:177-187): colours 0, 1, 0, 1 at the fine level
// (the first reads no z), 1, 0, 1 below it (the restriction wrote colour 0).
template <bool S, class ZT>
void vdown_t(const Ctx& c, cudaStream_t stream) {
    const Levels& V = c.lv;
    const int lc = V.lc;  // levels 0..lc-1 run per-level kernels, lc..L-1 the shared-memory group
    const int lgroup = V.lc;
    for (int l = 0; l < lc; l++) {
        const Lvl& L = V.lv[l];
        const Lvl& C = V.lv[l + 1];
        const int l0 = l == 0, first = l + 1 < lgroup;
        if (use_pair(c, l) && l == 0) {
            // colour 1 goes to zt, then back to z[1]
            launch_pair<HS_FIRST, HS_PLAIN, S, ZT>(c, L, C, l0, 0, L.zt, stream);
            launch_pair<HS_PLAIN, HS_PLAIN, S, ZT>(c, with_z(L, 1, L.zt), C, l0, 0, L.z[1], stream);
            launch_restrict<S, ZT>(c, L, C, l0, first, stream);
        } else if (use_pair(c, l)) {
            // colour 1 ends in zt (and stays there through the up sweeps)
            launch_hs<HS_PLAIN, S, ZT>(c, L, C, l0, 1, stream);
            launch_pair<HS_PLAIN, HS_PLAIN, S, ZT>(c, L, C, l0, 0, L.zt, stream);
            launch_restrict<S, ZT>(c, with_z(L, 1, L.zt), C, l0, first, stream);
        } else {
            if (l == 0) launch_hs<HS_FIRST, S, ZT>(c, L, C, l0, 0, stream);
            launch_hs<HS_PLAIN, S, ZT>(c, L, C, l0, 1, stream);
            launch_hs<HS_PLAIN, S, ZT>(c, L, C, l0, 0, stream);
            launch_hs<HS_PLAIN, S, ZT>(c, L, C, l0, 1, stream);
            launch_restrict<S, ZT>(c, L, C, l0, first, stream);
        }
    }
}

// the ascent of a V-cycle: levels lc-1..0 (prolongation and sweeps
// 1, 0, 1, 0, mgpcg.py:189-195); with final_zr the last sweep also forms z.r
// and the iteration's bookkeeping
template <bool S, class ZT>
void vup_t(const Ctx& c, cudaStream_t stream, bool final_zr) {
    const Levels& V = c.lv;
    const int lc = V.lc;
    for (int l = lc - 1; l >= 0; l--) {
        const Lvl& L = V.lv[l];
        const Lvl C = l + 1 < lc ? up_layout(c, l + 1) : V.lv[l + 1];
        const int l0 = l == 0;
        const bool zr = l == 0 && final_zr;
        if (use_pair(c, l) && l == 0) {
            // colour 0 goes to zt, then back to z[0]
            launch_pair<HS_PROLONG, HS_PLAIN, S, ZT>(c, L, C, l0, 1, L.zt, stream);
            if (zr) launch_pair<HS_PLAIN, HS_ZR, S, ZT>(c, with_z(L, 0, L.zt), C, l0, 1, L.z[0], stream);
            else launch_pair<HS_PLAIN, HS_PLAIN, S, ZT>(c, with_z(L, 0, L.zt), C, l0, 1, L.z[0], stream);
        } else if (use_pair(c, l)) {
            // colour 1 is in zt since the descent; colour 0 goes to z[1], then back to z[0]
            const Lvl Lx = with_z(L, 1, L.zt);
            launch_pair<HS_PROLONG, HS_PLAIN, S, ZT>(c, Lx, C, l0, 1, L.z[1], stream);
            launch_pair<HS_PLAIN, HS_PLAIN, S, ZT>(c, with_z(Lx, 0, L.z[1]), C, l0, 1, L.z[0], stream);
        } else {
            launch_hs<HS_PROLONG, S, ZT>(c, L, C, l0, 1, stream);
            launch_hs<HS_PLAIN, S, ZT>(c, L, C, l0, 0, stream);
            launch_hs<HS_PLAIN, S, ZT>(c, L, C, l0, 1, stream);
            if (zr) launch_hs<HS_ZR, S, ZT>(c, L, C, l0, 0, stream);
            else launch_hs<HS_PLAIN, S, ZT>(c, L, C, l0, 0, stream);
        }
    }
}


// One V-cycle (mgpcg.py:177-195); with final_zr the last kernel also forms
// z.r and the end-of-iteration bookkeeping (mgpcg.py:263-277).
template <bool S, class ZT>
void vcycle_t(const Ctx& c, cudaStream_t stream, bool final_zr) {
    const Levels& V = c.lv;
    const int lc = V.lc;
    vdown_t<S, ZT>(c, stream);
    if (final_zr && lc == 0) {
        launch_pdl(k_coarse<true, S, ZT>, 1, 1024, c.csmem, stream, c.g, V);
    } else {
        launch_pdl(k_coarse<false, S, ZT>, 1, 1024, c.csmem, stream, c.g, V);
    }
    vup_t<S, ZT>(c, stream, final_zr);
}

void enqueue_vcycle(const Ctx& c, bool solid, cudaStream_t stream, bool final_zr) {
    if (c.ztype == 1) {
        if (solid) vcycle_t<true, __nv_bfloat16>(c, stream, final_zr);
        else vcycle_t<false, __nv_bfloat16>(c, stream, final_zr);
    } else if (c.ztype == 2) {
        if (solid) vcycle_t<true, __half>(c, stream, final_zr);
        else vcycle_t<false, __half>(c, stream, final_zr);
    } else {
        if (solid) vcycle_t<true, float>(c, stream, final_zr);
        else vcycle_t<false, float>(c, stream, final_zr);
    }
}

template <bool S, class ZT>
void cg_kernels(const Ctx& c, cudaStream_t stream) {
    const Lvl& L = c.lv.lv[0];
    if (L.vec) {
        const int g = rgrid((long long)L.n0 * L.n1 * (L.H / 4));
        launch_pdl(k_cg_ap4<S, ZT>, g, 256, 0, stream, c.g, L, c.f);
        launch_pdl(k_cg_xr4<S>, g, 256, 0, stream, c.g, L, c.f);
    } else {
        launch_pdl(k_cg_ap<S, ZT>, rgrid(L.P), 256, 0, stream, c.g, L, c.f);
        launch_pdl(k_cg_xr<S>, rgrid(L.P), 256, 0, stream, c.g, L, c.f);
    }
}

// The body of one CG iteration (mgpcg.py:236-277), enqueued on `stream`.
void enqueue_cg(const Ctx& c, bool solid, cudaStream_t stream) {
    if (c.ztype == 1) {
        if (solid) cg_kernels<true, __nv_bfloat16>(c, stream);
        else cg_kernels<false, __nv_bfloat16>(c, stream);
    } else if (c.ztype == 2) {
        if (solid) cg_kernels<true, __half>(c, stream);
        else cg_kernels<false, __half>(c, stream);
    } else {
        if (solid) cg_kernels<true, float>(c, stream);
        else cg_kernels<false, float>(c, stream);
    }
}

// The stepwise solve on the per-level kernels: a V-cycle's descent, and one
// step = the ascent with z.r, the CG kernels, the next descent.
template <bool S, class ZT>
void step_pl_t(const Ctx& c, cudaStream_t stream, bool down_only) {
    if (!down_only) {
        vup_t<S, ZT>(c, stream, true);
        cg_kernels<S, ZT>(c, stream);
    }
    vdown_t<S, ZT>(c, stream);
}
void enqueue_step_pl(const Ctx& c, bool solid, cudaStream_t stream, bool down_only) {
    if (c.ztype == 1) {
        if (solid) step_pl_t<true, __nv_bfloat16>(c, stream, down_only);
        else step_pl_t<false, __nv_bfloat16>(c, stream, down_only);
    } else if (c.ztype == 2) {
        if (solid) step_pl_t<true, __half>(c, stream, down_only);
        else step_pl_t<false, __half>(c, stream, down_only);
    } else {
        if (solid) step_pl_t<true, float>(c, stream, down_only);
        else step_pl_t<false, float>(c, stream, down_only);
    }
}

void enqueue_iteration(const Ctx& c, bool solid, cudaStream_t stream) {
    enqueue_cg(c, solid, stream);
    enqueue_vcycle(c, solid, stream, true);
}

// set-up kernels of Poisson / solve (everything before the CG loop)
void enqueue_setup(Solver* s, Faces U, const float* rhs, double abs_tol, double rel_tol, int max_iters,
                   cudaStream_t cs, bool stepwise = false) {
    Ctx& c = s->ctx;
    const Lvl& L0 = c.lv.lv[0];
    int n = L0.n0 * L0.n1 * L0.n2;
    int nx = s->nx, ny = s->ny, nz = s->nz;
    if (!rhs) {
        const int plane = std::max(ny * nz, std::max(nx * nz, nx * ny));
        k_apply_walls<<<dim3(std::min(grid_for(plane), 1184), 6), 256, 0, cs>>>(c.g, nx, ny, nz, U);
        if (s->solid) k_apply_solid<<<grid_for(n), 256, 0, cs>>>(c.g.st, nx, ny, nz, L0.bm, s->bvel, U);
    }
    if (s->solid) {
        for (int l = 1; l < c.lv.L; l++) {
            const Lvl& F = c.lv.lv[l - 1];
            const Lvl& C = c.lv.lv[l];
            k_downsample_bm<<<grid_for((long long)C.n0 * C.n1 * C.n2), 256, 0, cs>>>(c.g.st, F.bm, C.bm, C.n0, C.n1,
                                                                                    C.n2, F.n1, F.n2);
        }
        for (int l = 0; l < c.lv.L; l++) {
            const Lvl& V = c.lv.lv[l];
            k_codes<<<rgrid((long long)V.n0 * V.n1 * V.n2), 256, 0, cs>>>(c.g, V);
        }
    }
    cudaMemsetAsync(c.g.st->counter, 0, sizeof(c.g.st->counter), cs);  // fresh reduction counters
    if (s->solid) k_setup_rhs<true><<<rgrid(L0.P), 256, 0, cs>>>(c.g, L0, c.f, U, rhs, abs_tol, rel_tol, max_iters);
    else k_setup_rhs<false><<<rgrid(L0.P), 256, 0, cs>>>(c.g, L0, c.f, U, rhs, abs_tol, rel_tol, max_iters);
    if (s->solid && !rhs) k_solid_fix<<<rgrid(L0.P), 256, 0, cs>>>(c.g, L0, c.f);
    if (stepwise) enqueue_step_pl(c, s->solid, cs, true);  // the stepwise solve: the first V-cycle's descent
    else enqueue_vcycle(c, s->solid, cs, true);          // first preconditioner application + z.r + tol
}

// gradient update (Poisson) or the solution copy (solve)
void enqueue_finish(Solver* s, Faces U, const float* rhs, float* xout, cudaStream_t cs) {
    Ctx& c = s->ctx;
    const Lvl& L0 = c.lv.lv[0];
    int n = L0.n0 * L0.n1 * L0.n2;
    int nx = s->nx, ny = s->ny, nz = s->nz;
    if (!rhs) {
        k_grad_p<<<rgrid(L0.P), 256, 0, cs>>>(c.g, L0, c.f, U);
        if (s->solid) k_apply_solid<<<grid_for(n), 256, 0, cs>>>(c.g.st, nx, ny, nz, L0.bm, s->bvel, U);
    } else {
        k_from_rb<<<rgrid(n), 256, 0, cs>>>(c.g.st, L0, c.f.x[0], c.f.x[1], xout, &c.g.st->x_valid, 0, nullptr);
    }
}

// set-up, then the conditional while node, then the gradient update; captured
// into a graph
int build_graph(Solver* s, Faces U, const float* rhs, float* xout, double abs_tol, double rel_tol, int max_iters,
                cudaGraphExec_t* exec) {
    cudaStream_t cs;
    CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t graph;
    CK(cudaGraphCreate(&graph, 0));
    cudaGraphConditionalHandle handle;
    CK(cudaGraphConditionalHandleCreate(&handle, graph, 0, cudaGraphCondAssignDefault));
    s->ctx.g.cond = handle;
    s->ctx.g.use_cond = 1;
    // 1) set-up
    CK(cudaStreamBeginCaptureToGraph(cs, graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    enqueue_setup(s, U, rhs, abs_tol, rel_tol, max_iters, cs);
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
    cudaGraph_t b2;
    //    the CG kernels, then if (still running) { V-cycle }: the V-cycle's
    //    kernels are captured with nochk (see stopped())
    cudaGraphConditionalHandle vh;
    CK(cudaGraphConditionalHandleCreate(&vh, body, 0, 0));
    s->ctx.g.vcond = vh;
    s->ctx.g.use_vcond = 1;
    CK(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    enqueue_cg(s->ctx, s->solid, cs);
    CK(cudaStreamEndCapture(cs, &b2));
    CK(cudaGraphGetNodes(body, nullptr, &nn));
    nodes.resize(nn);
    CK(cudaGraphGetNodes(body, nodes.data(), &nn));
    cudaGraphNode_t bleaf = nullptr;
    for (auto nd : nodes) {
        size_t nout = 0;
        CK(cudaGraphNodeGetDependentNodes(nd, nullptr, &nout));
        if (nout == 0) bleaf = nd;
    }
    cudaGraphNodeParams ip = {};
    ip.type = cudaGraphNodeTypeConditional;
    ip.conditional.handle = vh;
    ip.conditional.type = cudaGraphCondTypeIf;
    ip.conditional.size = 1;
    cudaGraphNode_t inode;
    CK(cudaGraphAddNode(&inode, body, &bleaf, 1, &ip));
    Ctx vc = s->ctx;
    vc.g.nochk = 1;
    CK(cudaStreamBeginCaptureToGraph(cs, ip.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                     cudaStreamCaptureModeThreadLocal));
    enqueue_vcycle(vc, s->solid, cs, true);
    CK(cudaStreamEndCapture(cs, &b2));
    s->ctx.g.use_vcond = 0;  // launches outside this graph set no IF condition
    // 3) finish
    CK(cudaStreamBeginCaptureToGraph(cs, graph, &cnode, nullptr, 1, cudaStreamCaptureModeThreadLocal));
    enqueue_finish(s, U, rhs, xout, cs);
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
    s->ctx.g.use_cond = 0;
    s->ctx.g.use_vcond = 0;
    enqueue_setup(s, U, rhs, abs_tol, rel_tol, max_iters, cs);
    for (int it = 0; it <= max_iters + 8; it++) {
        CK(cudaMemcpyAsync(&s->st_host->status, &s->ctx.g.st->status, sizeof(int), cudaMemcpyDeviceToHost, cs));
        CK(cudaStreamSynchronize(cs));
        if (s->st_host->status != ST_RUNNING) break;
        enqueue_iteration(s->ctx, s->solid, cs);
    }
    enqueue_finish(s, U, rhs, xout, cs);
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
    key.a[6] = rhs;
    key.a[7] = xout;
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

// the C-ABI code of a solve status
int status_code(int st) {
    switch (st) {
        case ST_CONVERGED: return EDGE_OK;
        case ST_NAN: return EDGE_ENAN;
        default: return EDGE_ENOCONV;
    }
}

// levels of a grid (mgpcg.py:34); EDGE_EINVAL when a level would not halve
int level_count(int nx, int ny, int nz, int base_level, int* L) {
    int mn = std::min(nx, std::min(ny, nz));
    int lg = 0;
    while ((1 << (lg + 1)) <= mn) lg++;
    *L = lg - base_level + 1;
    if (*L < 1 || *L > 16) return EDGE_EINVAL;
    for (int l = 1; l < *L; l++) {
        int f = 1 << l;
        // restrict writes r[l+1][I//2]: every level must halve exactly
        if (nx % f || ny % f || nz % f) return EDGE_EINVAL;
    }
    return EDGE_OK;
}

}  // namespace

extern "C" {

int edge_mgpcg_create(void** handle, int nx, int ny, int nz, int base_level, const int* bt, const int* mask,
                      const float* bvel, int precision) {
    if (!handle || !bt || nx < 2 || ny < 2 || nz < 2) return EDGE_EINVAL;
    if ((mask == nullptr) != (bvel == nullptr)) return EDGE_EINVAL;
    if (precision < 0 || precision > 2) return EDGE_EINVAL;
    long long n = (long long)nx * ny * nz;
    if (n * 3 >= (1LL << 31)) return EDGE_EINVAL;
    int L = 0;
    if (level_count(nx, ny, nz, base_level, &L) != EDGE_OK) return EDGE_EINVAL;
    Solver* s = new Solver();
    s->nx = nx; s->ny = ny; s->nz = nz;
    s->solid = mask != nullptr;
    s->bvel = bvel;
    s->precision = precision;
    Ctx& c = s->ctx;
    memset(&c, 0, sizeof(c));
    c.lv.L = L;
    c.ztype = precision;
    for (int q = 0; q < 6; q++) c.g.bt[q] = bt[q];
    c.g.walls = 0;
    for (int q = 0; q < 6; q++) c.g.walls |= (bt[q] == 2) << q;
    int r = EDGE_OK;
    for (int l = 0; l < L && r == EDGE_OK; l++) {
        Lvl& V = c.lv.lv[l];
        set_level_dims(V, nx >> l, ny >> l, nz >> l);
        size_t pa = plane_alloc(V.P);
        // level 0's r is the FP32 CG residual; the other level arrays are
        // BF16 in the mixed-precision solver
        const size_t esz = precision != 0 ? 2 : 4, esr = l == 0 ? 4 : esz;
        r = alloc(s, (void**)&V.r[0], 2 * pa * esr);
        if (r == EDGE_OK) r = alloc(s, (void**)&V.z[0], 2 * pa * esz);
        if (r == EDGE_OK) r = cu(cudaMemset(V.z[0], 0, 2 * pa * esz));
        V.r[1] = reinterpret_cast<float*>(reinterpret_cast<char*>(V.r[0]) + pa * esr);
        V.z[1] = reinterpret_cast<float*>(reinterpret_cast<char*>(V.z[0]) + pa * esz);
        if (s->solid && r == EDGE_OK) {
            if (l == 0) V.bm = const_cast<int*>(mask);
            else r = alloc(s, (void**)&V.bm, (size_t)V.n0 * V.n1 * V.n2 * sizeof(int));
            if (r == EDGE_OK) r = alloc(s, (void**)&V.code[0], 2 * pa * sizeof(unsigned short));
            V.code[1] = V.code[0] + pa;
        }
    }
    plan_coarse(c, s->solid);
    // the third z plane of each per-level V-cycle level (fused half-sweep pairs)
    for (int l = 0; l < c.lv.lc && r == EDGE_OK; l++) {
        Lvl& V = c.lv.lv[l];
        const size_t esz = precision != 0 ? 2 : 4;
        r = alloc(s, (void**)&V.zt, plane_alloc(V.P) * esz);
        if (r == EDGE_OK) r = cu(cudaMemset(V.zt, 0, plane_alloc(V.P) * esz));
    }
    if (r == EDGE_OK) r = prepare_coarse_kernels(c);
    const size_t pa0 = plane_alloc(c.lv.lv[0].P);
    if (r == EDGE_OK) r = alloc(s, (void**)&c.f.x[0], 2 * pa0 * sizeof(float));
    if (r == EDGE_OK) r = alloc(s, (void**)&c.f.p[0][0], 4 * pa0 * sizeof(float));
    if (r == EDGE_OK) r = alloc(s, (void**)&c.f.div, n * sizeof(float));
    if (r == EDGE_OK) r = cu(cudaMemset(c.f.div, 0, n * sizeof(float)));
    if (r == EDGE_OK) {
        c.f.x[1] = c.f.x[0] + pa0;
        c.f.p[0][1] = c.f.p[0][0] + pa0;
        c.f.p[1][0] = c.f.p[0][0] + 2 * pa0;
        c.f.p[1][1] = c.f.p[0][0] + 3 * pa0;
    }
    if (r == EDGE_OK) r = alloc(s, (void**)&c.g.partials, 4 * (size_t)(kMaxBlocks + 64) * sizeof(double));
    if (r == EDGE_OK) r = alloc(s, (void**)&c.g.st, sizeof(SolveState));
    if (r == EDGE_OK) {
        SolveState st;
        memset(&st, 0, sizeof(st));
        st.all_neumann = (bt[0] + bt[1] + bt[2] + bt[3] + bt[4] + bt[5]) == 12;
        st.zsc = st.zinv = 1.0f;
        st.zscaled = precision == 2;
        r = cu(cudaMemcpy(c.g.st, &st, sizeof(st), cudaMemcpyHostToDevice));
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

int edge_mgpcg_levels(void* handle) { return handle ? ((Solver*)handle)->ctx.lv.L : EDGE_EINVAL; }

int edge_mgpcg_kernel_count(void* handle, long long* count, void* stream) {
    if (!handle || !count) return EDGE_EINVAL;
    Solver* s = (Solver*)handle;
    CK(cudaMemcpyAsync(s->st_host, s->ctx.g.st, sizeof(SolveState), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
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
    CK(cudaMemcpyAsync(s->st_host, s->ctx.g.st, sizeof(SolveState), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    CK(cudaStreamSynchronize((cudaStream_t)stream));
    const SolveState& st = *s->st_host;
    if (iters) *iters = st.it;
    if (rTr) *rTr = st.rTr;
    if (status)
        *status = status_code(st.status);
    return EDGE_OK;
}

int edge_mgpcg_restart(void* handle, void* stream) {
    if (!handle) return EDGE_EINVAL;
    Solver* s = (Solver*)handle;
    k_set_restart<<<1, 32, 0, (cudaStream_t)stream>>>(s->ctx.g.st);
    return cu(cudaPeekAtLastError());
}

int edge_mgpcg_progress(void* handle, int* iters, double* rTr, int* running, void* stream) {
    if (!handle) return EDGE_EINVAL;
    Solver* s = (Solver*)handle;
    CK(cudaMemcpyAsync(s->st_host, s->ctx.g.st, sizeof(SolveState), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    CK(cudaStreamSynchronize((cudaStream_t)stream));
    if (iters) *iters = s->st_host->it;
    if (rTr) *rTr = s->st_host->rTr;
    if (running) *running = s->st_host->status == ST_RUNNING;
    return EDGE_OK;
}

int edge_mgpcg_vcycle(void* handle, const float* r, float* z, void* stream) {
    if (!handle || !r || !z) return EDGE_EINVAL;
    Solver* s = (Solver*)handle;
    cudaStream_t st = (cudaStream_t)stream;
    Ctx c = s->ctx;
    const Lvl& L0 = c.lv.lv[0];
    int n = L0.n0 * L0.n1 * L0.n2;
    // status = running, mean = 0, setup flag on so the z.r epilogue is inert
    SolveState* hs = s->st_host;
    CK(cudaMemcpyAsync(hs, c.g.st, sizeof(SolveState), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    hs->status = ST_RUNNING;
    hs->mean = 0.0f;
    hs->setup = 1;
    hs->max_iters = 1;
    hs->abs_tol = 0.0;
    hs->rel_tol = 0.0;
    CK(cudaMemcpyAsync(c.g.st, hs, sizeof(SolveState), cudaMemcpyHostToDevice, st));
    if (s->solid) {
        for (int l = 1; l < c.lv.L; l++) {
            const Lvl& F = c.lv.lv[l - 1];
            const Lvl& C = c.lv.lv[l];
            k_downsample_bm<<<grid_for((long long)C.n0 * C.n1 * C.n2), 256, 0, st>>>(c.g.st, F.bm, C.bm, C.n0, C.n1,
                                                                                    C.n2, F.n1, F.n2);
        }
        for (int l = 0; l < c.lv.L; l++) {
            const Lvl& V = c.lv.lv[l];
            k_codes<<<rgrid((long long)V.n0 * V.n1 * V.n2), 256, 0, st>>>(c.g, V);
        }
    }
    k_to_rb<<<rgrid(n), 256, 0, st>>>(L0, r, L0.r[0], L0.r[1], 0);
    if (c.ztype == 2) k_zscale<<<rgrid(L0.P), 256, 0, st>>>(c.g, L0);  // the input's scale
    // outside a graph there is no loop condition to set
    c.g.use_cond = 0;
    enqueue_vcycle(c, s->solid, st, false);
    k_from_rb<<<rgrid(n), 256, 0, st>>>(nullptr, L0, L0.z[0], L0.z[1], z, nullptr, c.ztype, &c.g.st->zinv);
    return cu(cudaPeekAtLastError());
}

int edge_mgpcg_apply_A_f64(void* handle, const double* p, double* Ap, void* stream) {
    if (!handle || !p || !Ap) return EDGE_EINVAL;
    Solver* s = (Solver*)handle;
    const Lvl& L = s->ctx.lv.lv[0];
    k_apply_A64<<<grid_for((long long)L.n0 * L.n1 * L.n2), 256, 0, (cudaStream_t)stream>>>(s->ctx.g, L, p, Ap);
    return cu(cudaPeekAtLastError());
}

// ---- stepwise solve with a replaceable coarse solver -------------------------
int edge_mgpcg_coarse_shape(void* handle, int* level, int* dims) {
    if (!handle || !level || !dims) return EDGE_EINVAL;
    Solver* s = (Solver*)handle;
    const Levels& V = s->ctx.lv;
    *level = V.lc;
    dims[0] = V.lv[V.lc].n0;
    dims[1] = V.lv[V.lc].n1;
    dims[2] = V.lv[V.lc].n2;
    return V.lc >= 1 ? EDGE_OK : EDGE_ESTATE;
}

int edge_mgpcg_coarse_get_r(void* handle, float* dense, void* stream) {
    if (!handle || !dense) return EDGE_EINVAL;
    Solver* s = (Solver*)handle;
    const Lvl& C = s->ctx.lv.lv[s->ctx.lv.lc];
    const long long n = (long long)C.n0 * C.n1 * C.n2;
    k_from_rb<<<rgrid(n), 256, 0, (cudaStream_t)stream>>>(nullptr, C, C.r[0], C.r[1], dense, nullptr, s->ctx.ztype,
                                                         nullptr);
    return cu(cudaPeekAtLastError());
}

int edge_mgpcg_coarse_set_z(void* handle, const float* dense, void* stream) {
    if (!handle || !dense) return EDGE_EINVAL;
    Solver* s = (Solver*)handle;
    const Lvl& C = s->ctx.lv.lv[s->ctx.lv.lc];
    const long long n = (long long)C.n0 * C.n1 * C.n2;
    k_to_rb<<<rgrid(n), 256, 0, (cudaStream_t)stream>>>(C, dense, C.z[0], C.z[1], s->ctx.ztype);
    return cu(cudaPeekAtLastError());
}

int edge_mgpcg_coarse_default(void* handle, void* stream) {
    if (!handle) return EDGE_EINVAL;
    Solver* s = (Solver*)handle;
    if (s->ctx.lv.lc < 1) return EDGE_ESTATE;
    Ctx c = s->ctx;
    c.g.use_cond = 0;
    const int t = c.ztype;
    cudaStream_t st = (cudaStream_t)stream;
    if (t == 1) {
        if (s->solid) launch_pdl(k_coarse<false, true, __nv_bfloat16>, 1, 1024, c.csmem, st, c.g, c.lv);
        else launch_pdl(k_coarse<false, false, __nv_bfloat16>, 1, 1024, c.csmem, st, c.g, c.lv);
    } else if (t == 2) {
        if (s->solid) launch_pdl(k_coarse<false, true, __half>, 1, 1024, c.csmem, st, c.g, c.lv);
        else launch_pdl(k_coarse<false, false, __half>, 1, 1024, c.csmem, st, c.g, c.lv);
    } else {
        if (s->solid) launch_pdl(k_coarse<false, true, float>, 1, 1024, c.csmem, st, c.g, c.lv);
        else launch_pdl(k_coarse<false, false, float>, 1, 1024, c.csmem, st, c.g, c.lv);
    }
    return cu(cudaPeekAtLastError());
}

int edge_mgpcg_solve_begin(void* handle, const float* b, double abs_tol, double rel_tol, int max_iters,
                           void* stream) {
    if (!handle || !b) return EDGE_EINVAL;
    Solver* s = (Solver*)handle;
    if (s->ctx.lv.lc < 1) return EDGE_ESTATE;
    if (max_iters < 0) max_iters = s->solid ? 100 : 400;
    Faces U = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
    s->ctx.g.use_cond = 0;
    s->ctx.g.use_vcond = 0;
    s->ctx.g.nochk = 0;
    enqueue_setup(s, U, b, abs_tol, rel_tol, max_iters, (cudaStream_t)stream, true);
    return cu(cudaPeekAtLastError());
}

int edge_mgpcg_poisson_begin(void* handle, float* ux, float* uy, float* uz, double abs_tol, double rel_tol,
                             int max_iters, void* stream) {
    if (!handle || !ux || !uy || !uz) return EDGE_EINVAL;
    Solver* s = (Solver*)handle;
    if (s->ctx.lv.lc < 1) return EDGE_ESTATE;
    if (max_iters < 0) max_iters = s->solid ? 100 : 400;
    Faces U = {{ux, uy, uz}, {nullptr, nullptr, nullptr}};
    s->ctx.g.use_cond = 0;
    s->ctx.g.use_vcond = 0;
    s->ctx.g.nochk = 0;
    enqueue_setup(s, U, nullptr, abs_tol, rel_tol, max_iters, (cudaStream_t)stream, true);
    return cu(cudaPeekAtLastError());
}

int edge_mgpcg_poisson_end(void* handle, float* ux, float* uy, float* uz, float* fx, float* fy, float* fz,
                           void* stream) {
    if (!handle || !ux || !uy || !uz) return EDGE_EINVAL;
    Solver* s = (Solver*)handle;
    Faces U = {{ux, uy, uz}, {fx, fy, fz}};
    enqueue_finish(s, U, nullptr, nullptr, (cudaStream_t)stream);
    return cu(cudaPeekAtLastError());
}

int edge_mgpcg_solve_iter(void* handle, void* stream) {
    if (!handle) return EDGE_EINVAL;
    Solver* s = (Solver*)handle;
    if (s->ctx.lv.lc < 1) return EDGE_ESTATE;
    Ctx c = s->ctx;
    c.g.use_cond = 0;
    c.g.use_vcond = 0;
    c.g.nochk = 0;
    enqueue_step_pl(c, s->solid, (cudaStream_t)stream, false);
    return cu(cudaPeekAtLastError());
}

int edge_mgpcg_solve_end(void* handle, const float* b, float* x, void* stream) {
    if (!handle || !b || !x) return EDGE_EINVAL;
    Solver* s = (Solver*)handle;
    Faces U = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
    enqueue_finish(s, U, b, x, (cudaStream_t)stream);
    return cu(cudaPeekAtLastError());
}

int edge_mgpcg_refine_residual(void* handle, const double* b, const double* x, float* r, double* sums,
                               void* stream) {
    if (!handle || !b || !x || !r || !sums) return EDGE_EINVAL;
    Solver* s = (Solver*)handle;
    const Lvl& L = s->ctx.lv.lv[0];
    k_refine_residual<<<rgrid((long long)L.n0 * L.n1 * L.n2), 256, 0, (cudaStream_t)stream>>>(s->ctx.g, L, b, x, r,
                                                                                            sums, 6);
    return cu(cudaPeekAtLastError());
}

int edge_mgpcg_refine_update(void* handle, double* x, const float* d, void* stream) {
    if (!handle || !x || !d) return EDGE_EINVAL;
    Solver* s = (Solver*)handle;
    const Lvl& L = s->ctx.lv.lv[0];
    const long long n = (long long)L.n0 * L.n1 * L.n2;
    k_refine_update<<<rgrid(n), 256, 0, (cudaStream_t)stream>>>(n, x, d);
    return cu(cudaPeekAtLastError());
}

int edge_mgpcg_apply_A(void* handle, const float* p, float* Ap, void* stream) {
    if (!handle || !p || !Ap) return EDGE_EINVAL;
    Solver* s = (Solver*)handle;
    const Lvl& L = s->ctx.lv.lv[0];
    k_apply_A<<<grid_for((long long)L.n0 * L.n1 * L.n2), 256, 0, (cudaStream_t)stream>>>(s->ctx.g, L, p, Ap);
    return cu(cudaPeekAtLastError());
}

int edge_mgpcg_get(void* handle, int which, float* dst, void* stream) {
    if (!handle || !dst) return EDGE_EINVAL;
    Solver* s = (Solver*)handle;
    const Lvl& L = s->ctx.lv.lv[0];
    size_t n = (size_t)L.n0 * L.n1 * L.n2;
    cudaStream_t st = (cudaStream_t)stream;
    if (which == 0) return cu(cudaMemcpyAsync(dst, s->ctx.f.div, n * sizeof(float), cudaMemcpyDeviceToDevice, st));
    if (which == 1) {
        k_from_rb<<<rgrid((long long)n), 256, 0, st>>>(nullptr, L, s->ctx.f.x[0], s->ctx.f.x[1], dst,
                                                      &s->ctx.g.st->x_valid, 0, nullptr);
        return cu(cudaPeekAtLastError());
    }
    return EDGE_EINVAL;
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
constexpr long long kNoAllocFloats = 8 * kNoAllocMaxCells + 4096;

static __device__ __align__(256) float g_noalloc_scratch[kNoAllocFloats];
static __device__ __align__(256) double g_noalloc_partials[4 * (kMaxBlocks + 64)];
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
// once per device (with that device current).  The lookup is serialised, so
// host threads whose first calls on a device coincide fill the entry once.
int noalloc_addrs(NoAllocAddrs** out) {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return EDGE_EINVAL;
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
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
    int L = 0;
    if (level_count(nx, ny, nz, base_level, &L) != EDGE_OK) return EDGE_EINVAL;
    if (max_iters < 0) max_iters = 400;
    NoAllocAddrs* A = nullptr;
    int r = noalloc_addrs(&A);
    if (r != EDGE_OK) return r;
    cudaStream_t cs = (cudaStream_t)stream;
    // carve the scratch: 256-byte aligned planes
    Solver s;  // host-side description only; its containers stay empty
    s.nx = nx; s.ny = ny; s.nz = nz;
    s.solid = false;
    s.bvel = nullptr;
    s.precision = 0;
    s.st_host = nullptr;
    Ctx& c = s.ctx;
    memset(&c, 0, sizeof(c));
    c.lv.L = L;
    for (int q = 0; q < 6; q++) c.g.bt[q] = bt[q];
    c.g.walls = 0;
    for (int q = 0; q < 6; q++) c.g.walls |= (bt[q] == 2) << q;
    long long off = 0;
    auto take = [&](long long count) {
        float* p = A->scratch + off;
        off += (count + 63) / 64 * 64;
        return p;
    };
    for (int l = 0; l < L; l++) {
        Lvl& V = c.lv.lv[l];
        set_level_dims(V, nx >> l, ny >> l, nz >> l);
        for (int q = 0; q < 2; q++) V.r[q] = take(V.P);
        for (int q = 0; q < 2; q++) V.z[q] = take(V.P);
    }
    const int P0 = c.lv.lv[0].P;
    for (int q = 0; q < 2; q++) c.f.x[q] = take(P0);
    for (int b = 0; b < 2; b++)
        for (int q = 0; q < 2; q++) c.f.p[b][q] = take(P0);
    c.f.div = take(n);
    if (off > kNoAllocFloats) return EDGE_EINVAL;
    c.g.partials = A->partials;
    c.g.st = A->state;
    c.g.use_cond = 0;
    plan_coarse(c, false);
    // third z planes for the fused half-sweep pairs, where the scratch has room
    long long extra = 0;
    for (int l = 0; l < c.lv.lc; l++) extra += (c.lv.lv[l].P + 63) / 64 * 64;
    if (off + extra <= kNoAllocFloats)
        for (int l = 0; l < c.lv.lc; l++) c.lv.lv[l].zt = take(c.lv.lv[l].P);
    r = prepare_coarse_kernels(c);
    if (r != EDGE_OK) return r;
    // the loop state starts clean on every call (the arrays keep the last
    // call's contents; the set-up and the first iteration overwrite what is read)
    SolveState init;
    memset(&init, 0, sizeof(init));
    init.all_neumann = (bt[0] + bt[1] + bt[2] + bt[3] + bt[4] + bt[5]) == 12;
    init.zsc = init.zinv = 1.0f;
    CK(cudaMemcpyAsync(c.g.st, &init, sizeof(init), cudaMemcpyHostToDevice, cs));
    Faces U = {{ux, uy, uz}, {nullptr, nullptr, nullptr}};
    enqueue_setup(&s, U, nullptr, abs_tol, rel_tol, max_iters, cs);
    int st_status = ST_RUNNING;
    for (int it = 0; it <= max_iters + 8; it++) {
        CK(cudaMemcpyAsync(&st_status, &c.g.st->status, sizeof(int), cudaMemcpyDeviceToHost, cs));
        CK(cudaStreamSynchronize(cs));
        if (st_status != ST_RUNNING) break;
        enqueue_iteration(c, false, cs);
    }
    enqueue_finish(&s, U, nullptr, nullptr, cs);
    CK(cudaPeekAtLastError());
    SolveState fin;
    CK(cudaMemcpyAsync(&fin, c.g.st, sizeof(fin), cudaMemcpyDeviceToHost, cs));
    CK(cudaStreamSynchronize(cs));
    if (iters) *iters = fin.it;
    if (rTr) *rTr = fin.rTr;
    if (status) *status = status_code(fin.status);
    return EDGE_OK;
}
