// Learned preconditioner (a 3-D U-Net, no reference counterpart): BF16
// tensor-core convolutions on tcgen05 with FP32 accumulators in TMEM, the
// network's other layers, their backward passes and the optimiser step.
// The network is assembled on the host (edgeb200/unet.py) from these kernels.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstdint>

#include "tc_common.cuh"

using namespace edge;

namespace {

constexpr int kMaxPolls = 1 << 22;  // bounded mbarrier waits (each poll suspends briefly)

// One-CTA GEMM D = A B^T through the tensor cores, to pin down the operand
// layouts.  mode 0: M = 128, A (128 x K) and B (N x K) row-major, staged
// K-major; mode 1: M = 64, A given as (K x 64) and B as (K x N), staged
// MN-major.  D is M x N (FP32, row-major).
__global__ void __launch_bounds__(128) k_tc_selftest(int mode, int N, int K, const __nv_bfloat16* __restrict__ A,
                                                     const __nv_bfloat16* __restrict__ B, float* __restrict__ D,
                                                     int* err) {
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tslot;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int M = mode == 0 ? 128 : 64;
    const uint32_t ncols = N <= 32 ? 32 : (N <= 64 ? 64 : (N <= 128 ? 128 : 256));
    uint8_t* sA = smem;
    uint8_t* sB = smem + (size_t)M * K * 2;
    const uint32_t lboA = (uint32_t)(M / 8) * 128, lboB = (uint32_t)(N / 8) * 128;
    if (warp == 0) tc::tmem_alloc(tc::smem_u32(&tslot), ncols);
    if (tid == 0) tc::mbar_init(tc::smem_u32(&mbar), 1);
    // stage the operands: element (row r, k) of a K-major operand sits at
    // (k/8)*LBO + (r/8)*128 + (r%8)*16 + (k%8)*2; of an MN-major one at
    // (k/8)*LBO + (r/8)*128 + (k%8)*16 + (r%8)*2
    for (int e = tid; e < M * K; e += blockDim.x) {
        int r, k;
        if (mode == 0) { r = e / K; k = e % K; }
        else { k = e / M; r = e % M; }
        size_t off = mode == 0 ? (size_t)(k / 8) * lboA + (r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2
                               : (size_t)(k / 8) * lboA + (r / 8) * 128 + (k % 8) * 16 + (r % 8) * 2;
        *reinterpret_cast<__nv_bfloat16*>(sA + off) = A[e];
    }
    for (int e = tid; e < N * K; e += blockDim.x) {
        int r, k;
        if (mode == 0) { r = e / K; k = e % K; }
        else { k = e / N; r = e % N; }
        size_t off = mode == 0 ? (size_t)(k / 8) * lboB + (r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2
                               : (size_t)(k / 8) * lboB + (r / 8) * 128 + (k % 8) * 16 + (r % 8) * 2;
        *reinterpret_cast<__nv_bfloat16*>(sB + off) = B[e];
    }
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tbase = tslot;
    if (tid == 0) {
        const uint32_t idesc = tc::idesc_bf16(M, N, mode == 1, mode == 1);
        for (int ks = 0; ks < K / 16; ks++) {
            uint64_t da = tc::sdesc(tc::smem_u32(sA) + ks * 2 * lboA, lboA, 128);
            uint64_t db = tc::sdesc(tc::smem_u32(sB) + ks * 2 * lboB, lboB, 128);
            tc::mma_bf16(tbase, da, db, idesc, ks > 0 ? 1u : 0u);
        }
        tc::commit(tc::smem_u32(&mbar));
    }
    bool ok = tc::mbar_wait(tc::smem_u32(&mbar), 0, kMaxPolls);
    if (!ok) {
        if (tid == 0) atomicExch(err, 1);
        tc::mbar_wait(tc::smem_u32(&mbar), 0, kMaxPolls);  // the MMAs must finish before TMEM is freed
    }
    tc::fence_after_sync();
    if (ok) {
        // M = 128: row 32w + lane; M = 64: rows 16w .. 16w+15 in lanes 0-15
        const int row = mode == 0 ? 32 * warp + lane : 16 * warp + lane;
        for (int c0 = 0; c0 < N; c0 += 16) {
            float v[16];
            tc::tmem_ld16(tbase + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, v);
            if (mode == 0 || lane < 16)
#pragma unroll
                for (int q = 0; q < 16; q++)
                    if (c0 + q < N) D[(size_t)row * N + c0 + q] = v[q];
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_free(tbase, ncols);
}

// ===========================================================================
// Activations
// ===========================================================================
// Activation tensors ("padded chunked"): a level of interior size X x Y x Z
// is stored with one zero voxel of padding on each side, padded linear index
// v = (x+1) Sx + (y+1) Sy + (z+1) with Sy = Z+2, Sx = (Y+2)(Z+2), and its
// channels in chunks of 8: element (chunk q, voxel v, channel j) at
// (q Lc + G + v) 8 + j.  G = Sx + Sy + 2 guard voxels before and after the
// padded volume keep every 3x3x3 neighbourhood of a 128-voxel tile inside
// the buffer; Lc = G + Vt + G with Vt = Vp rounded up to 128.  Everything
// that is not an interior voxel holds zero, so the tiles' zero padding is
// read straight from memory.  A UMMA core matrix of 8 consecutive voxels x 8
// channels is then 128 contiguous bytes (K-major for the convolution's A
// operand, MN-major for the weight gradient's operands).

// x / d for 0 <= x < 2^31 by multiply-high (Granlund & Montgomery 1994)
struct DivU {
    unsigned m;
    int s;
};

struct Geo {
    int X, Y, Z;            // interior
    int Sy, Sx, Vp, Vt, G;  // strides, padded volume, tiled volume, guard
    long long Lc;           // voxels per channel chunk
    DivU dSx, dSy;
    int ntiles;
};

inline DivU host_fdiv(unsigned d) {
    int l = 0;
    while ((1ull << l) < d) l++;
    unsigned long long m = ((1ull << 32) * ((1ull << l) - d)) / d + 1;
    return DivU{(unsigned)m, l};
}

inline Geo make_geo(int X, int Y, int Z) {
    Geo g;
    g.X = X; g.Y = Y; g.Z = Z;
    g.Sy = Z + 2;
    g.Sx = (Y + 2) * (Z + 2);
    g.Vp = (X + 2) * g.Sx;
    g.Vt = (g.Vp + 127) / 128 * 128;
    g.G = g.Sx + g.Sy + 2;
    g.Lc = (long long)g.G * 2 + g.Vt;
    g.dSx = host_fdiv((unsigned)g.Sx);
    g.dSy = host_fdiv((unsigned)g.Sy);
    g.ntiles = g.Vt / 128;
    return g;
}

EDGE_D int fdivg(int x, DivU f) { return (int)((__umulhi((unsigned)x, f.m) + (unsigned)x) >> f.s); }

// interior coordinates of padded voxel v (false for padding and the tail)
EDGE_D bool interior(const Geo& g, int v, int& x, int& y, int& z) {
    if (v < 0 || v >= g.Vp) return false;
    int px = fdivg(v, g.dSx);
    int rem = v - px * g.Sx;
    int py = fdivg(rem, g.dSy);
    int pz = rem - py * g.Sy;
    x = px - 1; y = py - 1; z = pz - 1;
    return x >= 0 && x < g.X && y >= 0 && y < g.Y && z >= 0 && z < g.Z;
}

EDGE_D size_t act_off(const Geo& g, int q, long long v) { return ((size_t)q * g.Lc + g.G + v) * 8; }
EDGE_D int pvox(const Geo& g, int x, int y, int z) { return (x + 1) * g.Sx + (y + 1) * g.Sy + (z + 1); }
EDGE_D int tap_off(const Geo& g, int t) { return (t / 9 - 1) * g.Sx + ((t / 3) % 3 - 1) * g.Sy + (t % 3 - 1); }

EDGE_D void unpack8(uint4 raw, float (&f)[8]) {
    const __nv_bfloat16* h = reinterpret_cast<const __nv_bfloat16*>(&raw);
#pragma unroll
    for (int j = 0; j < 8; j++) f[j] = __bfloat162float(h[j]);
}
EDGE_D uint4 pack8(const float (&f)[8]) {
    __align__(16) __nv_bfloat16 o[8];
#pragma unroll
    for (int j = 0; j < 8; j++) o[j] = __float2bfloat16_rn(f[j]);
    return *reinterpret_cast<const uint4*>(o);
}

#define GSTRIDE(t, n) for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < (n); \
                           t += (long long)gridDim.x * blockDim.x)

// ===========================================================================
// Tensor-core 3x3x3 convolution (forward and data gradient)
// ===========================================================================
// y = act(sum_i conv(x_i, W_i) + bias) for one or two inputs (the U-Net's skip
// connection is a second input of the same convolution, not a concatenated
// copy).  Weights are packed per input as [tap][Cin/8][Cout][8] bf16 (a
// K-major B operand per tap).  One tile = 128 consecutive padded voxels (the
// M rows); for each input and each x-offset dx the CTA stages the three
// dy-rows of 130 voxels (all channel chunks) and the nine taps' weights, and
// one thread issues 9 taps x Cin/16 MMAs into the FP32 TMEM accumulator
// (M = 128, N = Cout, K = 16 each); the A operand of tap (dy, dz) is the
// staged row of dy shifted by dz voxels (16 bytes).  The data gradient is the
// same kernel with transposed, tap-flipped weights.
struct ConvIn {
    const __nv_bfloat16* x;
    const __nv_bfloat16* w;
    int cin;
};

constexpr int kSeg = 130;  // voxels staged per row (tile + 1 on each side)
constexpr uint32_t kSegBytes = kSeg * 16;

// The convolution kernel.  Thread 0 stages, per phase (input, dx), one
// 2080-byte bulk copy per (dy, channel chunk) row and one for the phase's
// weights into a stage of shared memory (completion counted on an mbarrier
// with expect_tx) and issues the phase's MMAs from it.  The kernel can ring
// two stages (the next phase's copies landing while the MMAs read the
// other); the launch uses one, whose smaller footprint lets two to four
// times more blocks share an SM, which measured faster on every U-Net layer
// (forward at 256x128x128: 3.03 ms against 3.52 ms with two stages, 4.88 ms
// with the stages filled by the threads instead of the copy engine).
template <int COUT>
__global__ void __launch_bounds__(128) k_conv_bulk(Geo g, ConvIn in0, ConvIn in1, int nin,
                                                   const float* __restrict__ bias, int flags,
                                                   __nv_bfloat16* __restrict__ y, int* err, int nstage,
                                                   uint32_t stage_bytes) {
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t full[2], mdone[2], tdone, fin;
    __shared__ uint32_t tslot;
    __shared__ int s_bad;
    constexpr uint32_t NCOLS = COUT < 32 ? 32 : COUT;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nchmax = max(in0.cin, nin > 1 ? in1.cin : 0) / 8;
    const uint32_t wofs = 3u * nchmax * kSegBytes;
    if (warp == 0) tc::tmem_alloc(tc::smem_u32(&tslot), NCOLS);
    if (tid == 0) {
        for (int s = 0; s < 2; s++) {
            tc::mbar_init(tc::smem_u32(&full[s]), 1);
            tc::mbar_init(tc::smem_u32(&mdone[s]), 1);
        }
        tc::mbar_init(tc::smem_u32(&tdone), 1);
        tc::mbar_init(tc::smem_u32(&fin), 1);
        s_bad = 0;
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tbase = tslot;
    const uint32_t idesc = tc::idesc_bf16(128, COUT, false, false);
    const uint32_t sbase = tc::smem_u32(smem);
    const int nph = 3 * nin;
    // thread 0's copy issue for phase ph of tile into stage s
    auto issue = [&](int tile, int ph, int s) {
        const ConvIn in = ph >= 3 ? in1 : in0;
        const int nch = in.cin / 8, dxi = ph % 3;
        const uint32_t st = sbase + (uint32_t)s * stage_bytes, fb = tc::smem_u32(&full[s]);
        tc::mbar_expect_tx(fb, 3u * nch * kSegBytes + 9u * nch * COUT * 16);
        const long long base = (long long)tile * 128 + (dxi - 1) * (long long)g.Sx - g.Sy - 1;
        for (int dyi = 0; dyi < 3; dyi++)
            for (int q = 0; q < nch; q++)
                tc::bulk_g2s(st + (uint32_t)(dyi * nch + q) * kSegBytes, in.x + act_off(g, q, base + dyi * g.Sy),
                             kSegBytes, fb);
        tc::bulk_g2s(st + wofs, reinterpret_cast<const uint4*>(in.w) + (size_t)dxi * 9 * nch * COUT,
                     9u * nch * COUT * 16, fb);
    };
    uint32_t fpar[2] = {0, 0}, mpar[2] = {0, 0}, tpar = 0;
    bool inflight[2] = {false, false};  // thread 0: a stage's copies not yet waited for
    int n = 0;                          // thread 0: phases issued to the tensor cores so far
    bool bad = false;
    if (tid == 0 && (int)blockIdx.x < g.ntiles) {
        issue(blockIdx.x, 0, 0);
        inflight[0] = true;
    }
    for (int tile = blockIdx.x; tile < g.ntiles; tile += gridDim.x) {
        if (tid == 0) {
            int nmma = 0;
            for (int ph = 0; ph < nph; ph++, n++) {
                const int s = nstage == 2 ? (n & 1) : 0;
                if (!tc::mbar_wait(tc::smem_u32(&full[s]), fpar[s], kMaxPolls)) { s_bad = 1; break; }
                fpar[s] ^= 1;
                inflight[s] = false;
                tc::fence_after_sync();
                const int nch = (ph >= 3 ? in1.cin : in0.cin) / 8;
                const uint32_t a0 = sbase + (uint32_t)s * stage_bytes, b0 = a0 + wofs;
                for (int dyi = 0; dyi < 3; dyi++)
                    for (int dzi = 0; dzi < 3; dzi++)
                        for (int ks = 0; ks < nch / 2; ks++) {
                            const uint64_t da =
                                tc::sdesc(a0 + (uint32_t)((dyi * nch + 2 * ks) * kSegBytes + dzi * 16), kSegBytes, 128);
                            const uint64_t db =
                                tc::sdesc(b0 + (uint32_t)(((dyi * 3 + dzi) * nch + 2 * ks) * COUT * 16), COUT * 16, 128);
                            tc::mma_bf16(tbase, da, db, idesc, nmma > 0 ? 1u : 0u);
                            nmma++;
                        }
                tc::commit(tc::smem_u32(&mdone[s]));
                if (ph == nph - 1) tc::commit(tc::smem_u32(&tdone));
                // the next phase (of this tile, or the first of this block's next tile)
                int nt = tile, np = ph + 1;
                if (np == nph) { nt = tile + gridDim.x; np = 0; }
                if (nt < g.ntiles) {
                    const int s2 = nstage == 2 ? ((n + 1) & 1) : 0;
                    // the stage was last read by phase n - 1 (two stages) or n (one)
                    if (nstage == 1 || n >= 1) {
                        if (!tc::mbar_wait(tc::smem_u32(&mdone[s2]), mpar[s2], kMaxPolls)) { s_bad = 1; break; }
                        mpar[s2] ^= 1;
                    }
                    issue(nt, np, s2);
                    inflight[s2] = true;
                }
            }
        }
        __syncthreads();
        if (s_bad) { bad = true; break; }
        {
            bool ok = tc::mbar_wait(tc::smem_u32(&tdone), tpar, kMaxPolls);
            tpar ^= 1;
            if (__syncthreads_or(!ok)) { bad = true; break; }
        }
        tc::fence_after_sync();
        const int v0 = tile * 128;
        const int v = v0 + 32 * warp + lane;
        int x, yy, z;
        const bool in_dom = interior(g, v, x, yy, z);
#pragma unroll
        for (int c0 = 0; c0 < COUT; c0 += 16) {
            float acc[16];
            tc::tmem_ld16(tbase + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, acc);
#pragma unroll
            for (int h = 0; h < 2; h++) {
                uint4* dst = reinterpret_cast<uint4*>(y + act_off(g, (c0 >> 3) + h, v));
                float old[8] = {0, 0, 0, 0, 0, 0, 0, 0}, o[8];
                if (flags & 2) unpack8(*dst, old);
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    float t = acc[8 * h + j] + (bias ? bias[c0 + 8 * h + j] : 0.0f);
                    if (flags & 1) t = fmaxf(t, 0.0f);
                    t += old[j];
                    o[j] = in_dom ? t : 0.0f;
                }
                *dst = pack8(o);
            }
        }
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
    }
    if (bad && tid == 0) {
        atomicExch(err, 1);
        // the copies still in flight land, and every MMA issued completes, before
        // the block exits and frees its tensor memory (bounded waits)
        for (int s = 0; s < 2; s++)
            if (inflight[s]) tc::mbar_wait(tc::smem_u32(&full[s]), fpar[s], kMaxPolls);
        tc::commit(tc::smem_u32(&fin));
        tc::mbar_wait(tc::smem_u32(&fin), 0, kMaxPolls);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_free(tbase, NCOLS);
}

// ===========================================================================
// Tensor-core weight gradient
// ===========================================================================
// dW[co][ci][t] = sum over voxels v of d[v][co] x[v + off(t)][ci] (d: the
// layer's pre-activation gradient, Cout channels; x: its input, CIN
// channels).  M = 64 rows (co, zero chunks above Cout), N = CIN, K = voxels;
// both operands are MN-major straight from the staged activations: a core
// matrix is 8 consecutive voxels x one 8-channel chunk.  CTA (group, split)
// accumulates the taps of one tap group (9 taps of one dx, or 3 taps of one
// (dx, dy) when 9 x CIN columns exceed TMEM) over the tiles split, split + S,
// ... in TMEM (one CIN-column block per tap) and writes its partial sums to
// partial[split][tap][co][ci].
template <int CIN>
__global__ void __launch_bounds__(128) k_wgrad_tc(Geo g, const __nv_bfloat16* __restrict__ d, int cout,
                                                  const __nv_bfloat16* __restrict__ x, float* __restrict__ partial,
                                                  int* err) {
    constexpr int TPG = 9 * CIN <= 512 ? 9 : 3;
    constexpr int NDY = TPG == 9 ? 3 : 1;
    constexpr int NCH = CIN / 8;
    constexpr uint32_t NEED = TPG * CIN;
    constexpr uint32_t NCOLS = NEED <= 32 ? 32 : (NEED <= 64 ? 64 : (NEED <= 128 ? 128 : (NEED <= 256 ? 256 : 512)));
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tslot;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int gid = blockIdx.x, split = blockIdx.y, S = gridDim.y;
    const int dxi = TPG == 9 ? gid : gid / 3;
    const int dy_fixed = TPG == 9 ? 0 : gid % 3;
    uint8_t* sA = smem;                 // 8 chunks x 128 voxels x 16 bytes
    uint8_t* sB = smem + 8 * 2048;      // NDY x NCH x 130 voxels x 16 bytes
    const int cch = cout / 8;
    if (warp == 0) tc::tmem_alloc(tc::smem_u32(&tslot), NCOLS);
    if (tid == 0) tc::mbar_init(tc::smem_u32(&mbar), 1);
    for (int e = tid; e < (8 - cch) * 128; e += blockDim.x)
        reinterpret_cast<uint4*>(sA + (size_t)cch * 2048)[e] = make_uint4(0, 0, 0, 0);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tbase = tslot;
    const uint32_t idesc = tc::idesc_bf16(64, CIN, true, true);
    uint32_t parity = 0;
    bool bad = false, pending = false, any = false;
    for (int tile = split; tile < g.ntiles && !bad; tile += S) {
        const int v0 = tile * 128;
        if (pending) {
            bool ok = tc::mbar_wait(tc::smem_u32(&mbar), parity, kMaxPolls);
            parity ^= 1;
            pending = false;
            if (__syncthreads_or(!ok)) { bad = true; break; }
        }
        for (int e = tid; e < cch * 128; e += blockDim.x) {
            const int q = e >> 7, m = e & 127;
            *reinterpret_cast<uint4*>(sA + (size_t)q * 2048 + m * 16) =
                *reinterpret_cast<const uint4*>(d + act_off(g, q, v0 + m));
        }
        for (int e = tid; e < NDY * NCH * kSeg; e += blockDim.x) {
            const int dyl = e / (NCH * kSeg), rem = e - dyl * NCH * kSeg;
            const int q = rem / kSeg, s = rem - q * kSeg;
            const int dyi = TPG == 9 ? dyl : dy_fixed;
            const long long v = (long long)v0 + (dxi - 1) * (long long)g.Sx + (dyi - 1) * (long long)g.Sy - 1 + s;
            *reinterpret_cast<uint4*>(sB + ((size_t)(dyl * NCH + q) * kSeg + s) * 16) =
                *reinterpret_cast<const uint4*>(x + act_off(g, q, v));
        }
        tc::fence_smem_to_async();
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (tid == 0) {
            const uint32_t a0 = tc::smem_u32(sA), b0 = tc::smem_u32(sB);
            for (int tl = 0; tl < TPG; tl++) {
                const int dyl = TPG == 9 ? tl / 3 : 0, dzi = tl % 3;
                for (int ks = 0; ks < 8; ks++) {
                    const uint64_t da = tc::sdesc(a0 + ks * 256, 128, 2048);
                    const uint64_t db =
                        tc::sdesc(b0 + (uint32_t)(dyl * NCH) * kSegBytes + dzi * 16 + ks * 256, 128, kSegBytes);
                    tc::mma_bf16(tbase + (uint32_t)(tl * CIN), da, db, idesc, (any || ks > 0) ? 1u : 0u);
                }
            }
            tc::commit(tc::smem_u32(&mbar));
        }
        pending = true;
        any = true;
    }
    if (pending && !bad) {
        bool ok = tc::mbar_wait(tc::smem_u32(&mbar), parity, kMaxPolls);
        parity ^= 1;
        if (__syncthreads_or(!ok)) bad = true;
    }
    if (!bad) {
        tc::fence_after_sync();
        const int co = 16 * warp + lane;
        for (int tl = 0; tl < TPG; tl++) {
            const int dyi = TPG == 9 ? tl / 3 : dy_fixed, dzi = tl % 3;
            const int tap = dxi * 9 + dyi * 3 + dzi;
            for (int c0 = 0; c0 < CIN; c0 += 16) {
                float v[16];
                tc::tmem_ld16(tbase + ((uint32_t)(32 * warp) << 16) + (uint32_t)(tl * CIN + c0), v);
                if (lane < 16 && co < cout)
#pragma unroll
                    for (int j = 0; j < 16; j++)
                        partial[(((size_t)split * 27 + tap) * cout + co) * CIN + c0 + j] = any ? v[j] : 0.0f;
            }
        }
    } else {
        if (tid == 0) atomicExch(err, 1);
        tc::mbar_wait(tc::smem_u32(&mbar), parity, kMaxPolls);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_free(tbase, NCOLS);
}

// dW[co][ci][t] = sum over splits (fixed order) of the partial sums
__global__ void k_reduce_wgrad(const float* __restrict__ partial, int S, int cout, int cin, float* __restrict__ dw) {
    GSTRIDE(e, (long long)cout * cin * 27) {
        const int t = (int)(e % 27), ci = (int)((e / 27) % cin), co = (int)(e / (27 * cin));
        float s = 0.0f;
        for (int k = 0; k < S; k++) s += partial[(((size_t)k * 27 + t) * cout + co) * cin + ci];
        dw[e] = s;
    }
}

// ===========================================================================
// SIMT layers: first (1 -> 16) and last (16 -> 1) convolutions, pooling,
// upsampling, and their backward passes
// ===========================================================================
// first: input r (float32, lexicographic interior grid) scaled by s; weights
// [16][27] already bf16-rounded (float), bias [16]; ReLU; bf16 output
__global__ void __launch_bounds__(256) k_conv_first(Geo g, const float* __restrict__ r, const float* __restrict__ scale,
                                                    const float* __restrict__ w, const float* __restrict__ bias,
                                                    __nv_bfloat16* __restrict__ y) {
    const int n = g.X * g.Y * g.Z;
    const float s = *scale;
    // the weights tap-major in shared memory: one tap's 16 outputs are four
    // broadcast 16-byte loads
    __shared__ __align__(16) float ws[27 * 16];
    for (int e = threadIdx.x; e < 27 * 16; e += blockDim.x) ws[e] = w[(e % 16) * 27 + e / 16];
    __syncthreads();
    GSTRIDE(t, n) {
        const int z = (int)(t % g.Z), yy = (int)((t / g.Z) % g.Y), x = (int)(t / ((long long)g.Y * g.Z));
        float acc[16];
#pragma unroll
        for (int co = 0; co < 16; co++) acc[co] = 0.0f;
#pragma unroll 1
        for (int tap = 0; tap < 27; tap++) {
            const int a = x + tap / 9 - 1, b = yy + (tap / 3) % 3 - 1, c = z + tap % 3 - 1;
            const bool ok = a >= 0 && a < g.X && b >= 0 && b < g.Y && c >= 0 && c < g.Z;
            const float in = ok ? r[((size_t)a * g.Y + b) * g.Z + c] * s : 0.0f;
            const float4* wt = reinterpret_cast<const float4*>(ws + tap * 16);
#pragma unroll
            for (int c4 = 0; c4 < 4; c4++) {
                const float4 wv = wt[c4];
                acc[4 * c4 + 0] = fmaf(wv.x, in, acc[4 * c4 + 0]);
                acc[4 * c4 + 1] = fmaf(wv.y, in, acc[4 * c4 + 1]);
                acc[4 * c4 + 2] = fmaf(wv.z, in, acc[4 * c4 + 2]);
                acc[4 * c4 + 3] = fmaf(wv.w, in, acc[4 * c4 + 3]);
            }
        }
        const int v = pvox(g, x, yy, z);
#pragma unroll
        for (int q = 0; q < 2; q++) {
            float o[8];
#pragma unroll
            for (int j = 0; j < 8; j++) o[j] = fmaxf(acc[8 * q + j] + bias[8 * q + j], 0.0f);
            *reinterpret_cast<uint4*>(y + act_off(g, q, v)) = pack8(o);
        }
    }
}

// last: z = (sum over 27 taps x 16 channels of w * f0 + bias) / s, float32
// lexicographic output (no activation)
__global__ void __launch_bounds__(256) k_conv_last(Geo g, const __nv_bfloat16* __restrict__ f,
                                                   const float* __restrict__ w, const float* __restrict__ bias,
                                                   const float* __restrict__ scale, float* __restrict__ z) {
    const int n = g.X * g.Y * g.Z;
    const float inv = 1.0f / *scale;
    __shared__ __align__(16) float ws[27 * 16];  // tap-major, as in k_conv_first
    for (int e = threadIdx.x; e < 27 * 16; e += blockDim.x) ws[e] = w[(e % 16) * 27 + e / 16];
    __syncthreads();
    GSTRIDE(t, n) {
        const int zz = (int)(t % g.Z), yy = (int)((t / g.Z) % g.Y), x = (int)(t / ((long long)g.Y * g.Z));
        const int v = pvox(g, x, yy, zz);
        float acc = 0.0f;
#pragma unroll 1
        for (int tap = 0; tap < 27; tap++) {
            const int off = tap_off(g, tap);
            const float4* wt = reinterpret_cast<const float4*>(ws + tap * 16);
#pragma unroll
            for (int q = 0; q < 2; q++) {
                float h[8];
                unpack8(*reinterpret_cast<const uint4*>(f + act_off(g, q, v + off)), h);
                const float4 wa = wt[2 * q], wb = wt[2 * q + 1];
                const float wv[8] = {wa.x, wa.y, wa.z, wa.w, wb.x, wb.y, wb.z, wb.w};
#pragma unroll
                for (int j = 0; j < 8; j++) acc = fmaf(wv[j], h[j], acc);
            }
        }
        z[t] = (acc + bias[0]) * inv;
    }
}

// data gradient of the last layer: df0[u][ci] = sum_t w[ci][t] dzn[u - off(t)]
__global__ void __launch_bounds__(256) k_last_bwd_data(Geo g, const float* __restrict__ dzn,
                                                       const float* __restrict__ w, __nv_bfloat16* __restrict__ df) {
    const int n = g.X * g.Y * g.Z;
    GSTRIDE(t, n) {
        const int z = (int)(t % g.Z), yy = (int)((t / g.Z) % g.Y), x = (int)(t / ((long long)g.Y * g.Z));
        float acc[16];
#pragma unroll
        for (int c = 0; c < 16; c++) acc[c] = 0.0f;
#pragma unroll 1
        for (int tap = 0; tap < 27; tap++) {
            const int a = x - (tap / 9 - 1), b = yy - ((tap / 3) % 3 - 1), c = z - (tap % 3 - 1);
            if (a < 0 || a >= g.X || b < 0 || b >= g.Y || c < 0 || c >= g.Z) continue;
            const float dv = dzn[((size_t)a * g.Y + b) * g.Z + c];
#pragma unroll
            for (int ci = 0; ci < 16; ci++) acc[ci] = fmaf(__ldg(w + ci * 27 + tap), dv, acc[ci]);
        }
        const int v = pvox(g, x, yy, z);
#pragma unroll
        for (int q = 0; q < 2; q++) {
            float o[8];
#pragma unroll
            for (int j = 0; j < 8; j++) o[j] = acc[8 * q + j];
            *reinterpret_cast<uint4*>(df + act_off(g, q, v)) = pack8(o);
        }
    }
}

// 16 per-thread sums -> one block sum each (256 threads)
EDGE_D void block_sum16(float (&acc)[16], float* out) {
    __shared__ float sm[8][16];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < 16; c++)
        for (int o = 16; o > 0; o >>= 1) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
    if (lane == 0)
#pragma unroll
        for (int c = 0; c < 16; c++) sm[w][c] = acc[c];
    __syncthreads();
    if (threadIdx.x < 16) {
        float s = 0.0f;
        for (int k = 0; k < 8; k++) s += sm[k][threadIdx.x];
        out[threadIdx.x] = s;
    }
}

// weight gradient of the first layer: dW[co][t] = sum_v d[v][co] (s r)[v + off(t)]
// block (tap, b) -> partial[(tap * nblk + b) * 16 + co]
__global__ void __launch_bounds__(256) k_wgrad_first(Geo g, const __nv_bfloat16* __restrict__ d,
                                                     const float* __restrict__ r, const float* __restrict__ scale,
                                                     float* __restrict__ partial) {
    const int tap = blockIdx.x, nblk = gridDim.y;
    const int n = g.X * g.Y * g.Z;
    const float s = *scale;
    const int ddx = tap / 9 - 1, ddy = (tap / 3) % 3 - 1, ddz = tap % 3 - 1;
    float acc[16];
#pragma unroll
    for (int c = 0; c < 16; c++) acc[c] = 0.0f;
    for (long long t = (long long)blockIdx.y * blockDim.x + threadIdx.x; t < n; t += (long long)nblk * blockDim.x) {
        const int z = (int)(t % g.Z), yy = (int)((t / g.Z) % g.Y), x = (int)(t / ((long long)g.Y * g.Z));
        const int a = x + ddx, b = yy + ddy, c = z + ddz;
        if (a < 0 || a >= g.X || b < 0 || b >= g.Y || c < 0 || c >= g.Z) continue;
        const float xv = r[((size_t)a * g.Y + b) * g.Z + c] * s;
        const int v = pvox(g, x, yy, z);
#pragma unroll
        for (int q = 0; q < 2; q++) {
            float h[8];
            unpack8(*reinterpret_cast<const uint4*>(d + act_off(g, q, v)), h);
#pragma unroll
            for (int j = 0; j < 8; j++) acc[8 * q + j] = fmaf(h[j], xv, acc[8 * q + j]);
        }
    }
    block_sum16(acc, partial + ((size_t)tap * nblk + blockIdx.y) * 16);
}

// weight gradient of the last layer: dW[ci][t] = sum_v dzn[v] f0[v + off(t)][ci]
__global__ void __launch_bounds__(256) k_wgrad_last(Geo g, const float* __restrict__ dzn,
                                                    const __nv_bfloat16* __restrict__ f, float* __restrict__ partial) {
    const int tap = blockIdx.x, nblk = gridDim.y;
    const int n = g.X * g.Y * g.Z;
    const int off = tap_off(g, tap);
    float acc[16];
#pragma unroll
    for (int c = 0; c < 16; c++) acc[c] = 0.0f;
    for (long long t = (long long)blockIdx.y * blockDim.x + threadIdx.x; t < n; t += (long long)nblk * blockDim.x) {
        const int z = (int)(t % g.Z), yy = (int)((t / g.Z) % g.Y), x = (int)(t / ((long long)g.Y * g.Z));
        const float dv = dzn[t];
        const int v = pvox(g, x, yy, z) + off;
#pragma unroll
        for (int q = 0; q < 2; q++) {
            float h[8];
            unpack8(*reinterpret_cast<const uint4*>(f + act_off(g, q, v)), h);
#pragma unroll
            for (int j = 0; j < 8; j++) acc[8 * q + j] = fmaf(h[j], dv, acc[8 * q + j]);
        }
    }
    block_sum16(acc, partial + ((size_t)tap * nblk + blockIdx.y) * 16);
}

// out[c * 27 + t] = sum_b partial[(t * nblk + b) * 16 + c]
__global__ void k_reduce_taps16(const float* __restrict__ partial, int nblk, float* __restrict__ out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 16 * 27) return;
    const int c = e / 27, t = e % 27;
    float s = 0.0f;
    for (int b = 0; b < nblk; b++) s += partial[((size_t)t * nblk + b) * 16 + c];
    out[e] = s;
}

// per-channel sums of an activation tensor (bias gradients): block (q, b)
// sums chunk q over its share of voxels -> partial[(q * nblk + b) * 8 + j]
__global__ void __launch_bounds__(256) k_chan_sum(long long lc, const __nv_bfloat16* __restrict__ d,
                                                  float* __restrict__ partial) {
    const int q = blockIdx.x, nblk = gridDim.y;
    float acc[16];
#pragma unroll
    for (int c = 0; c < 16; c++) acc[c] = 0.0f;
    for (long long v = (long long)blockIdx.y * blockDim.x + threadIdx.x; v < lc; v += (long long)nblk * blockDim.x) {
        float h[8];
        unpack8(*reinterpret_cast<const uint4*>(d + ((size_t)q * lc + v) * 8), h);
#pragma unroll
        for (int j = 0; j < 8; j++) acc[j] += h[j];
    }
    __shared__ float res[16];
    block_sum16(acc, res);
    __syncthreads();
    if (threadIdx.x < 8) partial[((size_t)q * nblk + blockIdx.y) * 8 + threadIdx.x] = res[threadIdx.x];
}

__global__ void k_reduce_chan(const float* __restrict__ partial, int nblk, int C, float* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    float s = 0.0f;
    for (int b = 0; b < nblk; b++) s += partial[((size_t)(c / 8) * nblk + b) * 8 + (c % 8)];
    out[c] = s;
}

// out = dy where y > 0, else 0 (ReLU backward), on whole tensors
__global__ void __launch_bounds__(256) k_relu_bwd(long long n8, const __nv_bfloat16* __restrict__ dy,
                                                  const __nv_bfloat16* __restrict__ y, __nv_bfloat16* __restrict__ out) {
    GSTRIDE(e, n8) {
        float a[8], b[8];
        unpack8(reinterpret_cast<const uint4*>(dy)[e], a);
        unpack8(reinterpret_cast<const uint4*>(y)[e], b);
#pragma unroll
        for (int j = 0; j < 8; j++) a[j] = b[j] > 0.0f ? a[j] : 0.0f;
        reinterpret_cast<uint4*>(out)[e] = pack8(a);
    }
}

// ---- 2x2x2 mean pooling and nearest 2x upsampling (nch chunks of 8) ---------
__global__ void __launch_bounds__(256) k_pool(Geo gf, Geo gc, int nch, const __nv_bfloat16* __restrict__ fine,
                                              __nv_bfloat16* __restrict__ coarse) {
    const long long n = (long long)gc.X * gc.Y * gc.Z;
    GSTRIDE(t, n * nch) {
        const int q = (int)(t / n);
        const long long c = t - q * n;
        const int Z = (int)(c % gc.Z), Y = (int)((c / gc.Z) % gc.Y), X = (int)(c / ((long long)gc.Y * gc.Z));
        float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int a = 0; a < 8; a++) {
            float h[8];
            unpack8(*reinterpret_cast<const uint4*>(
                        fine + act_off(gf, q, pvox(gf, 2 * X + (a >> 2), 2 * Y + ((a >> 1) & 1), 2 * Z + (a & 1)))),
                    h);
#pragma unroll
            for (int j = 0; j < 8; j++) acc[j] += h[j];
        }
#pragma unroll
        for (int j = 0; j < 8; j++) acc[j] *= 0.125f;
        *reinterpret_cast<uint4*>(coarse + act_off(gc, q, pvox(gc, X, Y, Z))) = pack8(acc);
    }
}

// pooling backward: dfine = dcoarse / 8 (added to dfine when accum)
__global__ void __launch_bounds__(256) k_pool_bwd(Geo gf, Geo gc, int nch, const __nv_bfloat16* __restrict__ dcoarse,
                                                  __nv_bfloat16* __restrict__ dfine, int accum) {
    const long long n = (long long)gf.X * gf.Y * gf.Z;
    GSTRIDE(t, n * nch) {
        const int q = (int)(t / n);
        const long long c = t - q * n;
        const int z = (int)(c % gf.Z), y = (int)((c / gf.Z) % gf.Y), x = (int)(c / ((long long)gf.Y * gf.Z));
        float a[8], b[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        unpack8(*reinterpret_cast<const uint4*>(dcoarse + act_off(gc, q, pvox(gc, x / 2, y / 2, z / 2))), a);
        uint4* dst = reinterpret_cast<uint4*>(dfine + act_off(gf, q, pvox(gf, x, y, z)));
        if (accum) unpack8(*dst, b);
#pragma unroll
        for (int j = 0; j < 8; j++) a[j] = a[j] * 0.125f + b[j];
        *dst = pack8(a);
    }
}

__global__ void __launch_bounds__(256) k_upsample(Geo gc, Geo gf, int nch, const __nv_bfloat16* __restrict__ coarse,
                                                  __nv_bfloat16* __restrict__ fine) {
    const long long n = (long long)gf.X * gf.Y * gf.Z;
    GSTRIDE(t, n * nch) {
        const int q = (int)(t / n);
        const long long c = t - q * n;
        const int z = (int)(c % gf.Z), y = (int)((c / gf.Z) % gf.Y), x = (int)(c / ((long long)gf.Y * gf.Z));
        *reinterpret_cast<uint4*>(fine + act_off(gf, q, pvox(gf, x, y, z))) =
            *reinterpret_cast<const uint4*>(coarse + act_off(gc, q, pvox(gc, x / 2, y / 2, z / 2)));
    }
}

// upsampling backward: dcoarse = sum of the 8 children's gradients
__global__ void __launch_bounds__(256) k_up_bwd(Geo gc, Geo gf, int nch, const __nv_bfloat16* __restrict__ dfine,
                                                __nv_bfloat16* __restrict__ dcoarse) {
    const long long n = (long long)gc.X * gc.Y * gc.Z;
    GSTRIDE(t, n * nch) {
        const int q = (int)(t / n);
        const long long c = t - q * n;
        const int Z = (int)(c % gc.Z), Y = (int)((c / gc.Z) % gc.Y), X = (int)(c / ((long long)gc.Y * gc.Z));
        float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int a = 0; a < 8; a++) {
            float h[8];
            unpack8(*reinterpret_cast<const uint4*>(
                        dfine + act_off(gf, q, pvox(gf, 2 * X + (a >> 2), 2 * Y + ((a >> 1) & 1), 2 * Z + (a & 1)))),
                    h);
#pragma unroll
            for (int j = 0; j < 8; j++) acc[j] += h[j];
        }
        *reinterpret_cast<uint4*>(dcoarse + act_off(gc, q, pvox(gc, X, Y, Z))) = pack8(acc);
    }
}

// ---- weights, input scale, loss, optimiser -----------------------------------
// fp32 [Co][Ci][27] -> bf16 [27][Ci/8][Co][8] (forward), or for the data
// gradient the transposed, tap-flipped [27][Co/8][Ci][8] holding W[co][ci][26-t]
__global__ void k_pack_weights(const float* __restrict__ w, int co, int ci, int transpose,
                               __nv_bfloat16* __restrict__ out) {
    const int n = co * ci * 27;
    GSTRIDE(e, n) {
        // e enumerates the packed layout: ((t * kin/8 + q) * rows + row) * 8 + j
        const int rows = transpose ? ci : co, kin = transpose ? co : ci;
        const int j = (int)(e % 8), row = (int)((e / 8) % rows), q = (int)((e / (8 * rows)) % (kin / 8));
        const int t = (int)(e / ((long long)rows * kin));
        const int k = 8 * q + j;
        float v;
        if (transpose) v = w[((size_t)k * ci + row) * 27 + (26 - t)];  // row = ci, k = co
        else v = w[((size_t)row * ci + k) * 27 + t];                   // row = co, k = ci
        out[e] = __float2bfloat16_rn(v);
    }
}

// the scale 1/rms(r) of the network input: per-block float64 partial sums,
// the last block to finish (arrival counter) adds them in block order
__global__ void __launch_bounds__(256) k_input_scale(const float* __restrict__ r, long long n, double* partial,
                                                     unsigned* counter, float* scale) {
    __shared__ double sm[8];
    __shared__ bool last;
    double s = 0.0;
    GSTRIDE(e, n) s += (double)r[e] * (double)r[e];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; w++) t += sm[w];
        partial[blockIdx.x] = t;
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        double t = 0.0;
        for (unsigned b = 0; b < gridDim.x; b++) t += __ldcg(partial + b);
        *scale = (float)(1.0 / sqrt(t / (double)n));
        *counter = 0;
    }
}

// loss on the scaled problem: d = (z - target) s (z = network output / s);
// L = mean((d - mean d)^2), dL/dz_n = 2 (d - mean d) / n.  One block.
__global__ void __launch_bounds__(1024) k_loss_stats(const float* __restrict__ z, const float* __restrict__ x,
                                                     const float* __restrict__ scale, long long n,
                                                     double* __restrict__ stats) {
    __shared__ double sm[2][32];
    const double s = *scale;
    double a = 0.0, b = 0.0;
    for (long long e = threadIdx.x; e < n; e += blockDim.x) {
        double d = ((double)z[e] - (double)x[e]) * s;
        a += d;
        b += d * d;
    }
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if ((threadIdx.x & 31) == 0) { sm[0][threadIdx.x >> 5] = a; sm[1][threadIdx.x >> 5] = b; }
    __syncthreads();
    if (threadIdx.x < 32) {
        double ta = threadIdx.x < (blockDim.x >> 5) ? sm[0][threadIdx.x] : 0.0;
        double tb = threadIdx.x < (blockDim.x >> 5) ? sm[1][threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            ta += __shfl_xor_sync(0xffffffffu, ta, o);
            tb += __shfl_xor_sync(0xffffffffu, tb, o);
        }
        if (threadIdx.x == 0) {
            const double mean = ta / (double)n;
            stats[0] = mean;
            stats[1] = tb / (double)n - mean * mean;  // the loss
        }
    }
}

__global__ void __launch_bounds__(256) k_loss_grad(const float* __restrict__ z, const float* __restrict__ x,
                                                   const float* __restrict__ scale, const double* __restrict__ stats,
                                                   long long n, float* __restrict__ dzn) {
    const double s = *scale, mean = stats[0];
    GSTRIDE(e, n) dzn[e] = (float)(2.0 * (((double)z[e] - (double)x[e]) * s - mean) / (double)n);
}

// Adam (Kingma & Ba 2015): m = b1 m + (1-b1) g, v = b2 v + (1-b2) g^2,
// p -= lr (m / (1 - b1^t)) / (sqrt(v / (1 - b2^t)) + eps)
__global__ void __launch_bounds__(256) k_adam(long long n, float* __restrict__ p, const float* __restrict__ gr,
                                              float* __restrict__ m, float* __restrict__ v, float lr, float b1,
                                              float b2, float eps, float bc1, float bc2) {
    GSTRIDE(e, n) {
        const float g = gr[e];
        const float mm = b1 * m[e] + (1.0f - b1) * g;
        const float vv = b2 * v[e] + (1.0f - b2) * g * g;
        m[e] = mm;
        v[e] = vv;
        p[e] -= lr * (mm / bc1) / (sqrtf(vv / bc2) + eps);
    }
}

inline int g_sms() {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    return sms;
}

inline int cgrid(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148 * 16)); }
inline int rc_last() {
    cudaError_t e = cudaPeekAtLastError();
    return e == cudaSuccess ? EDGE_OK : (int)e;
}

// Blocks of a 128-thread convolution kernel with `smem` bytes of dynamic
// shared memory resident on one SM at once, with the kernel's carveout set to
// the maximum (228 KB per SM, of which each block also takes 1 KB reserved
// and a little static memory), at most the blocks whose tensor-memory
// columns fit in the SM's 512.  The kernels loop over tiles, so a grid of
// exactly this many blocks per SM runs in one wave (one block more per SM
// than fits would run as a nearly empty second wave).
static int resident_blocks(size_t smem, int cout) {
    const size_t per_block = smem + 1024 + 128;
    const int by_smem = (int)((size_t)228 * 1024 / per_block);
    const int by_tmem = 512 / (cout < 32 ? 32 : cout);
    return std::max(1, std::min(by_smem, by_tmem));
}

template <int COUT>
int launch_conv(const Geo& g, ConvIn a, ConvIn b, int nin, const float* bias, int flags, __nv_bfloat16* y, int* err,
                cudaStream_t st) {
    const int nchmax = std::max(a.cin, nin > 1 ? b.cin : 0) / 8;
    const size_t smem = (size_t)3 * nchmax * kSegBytes + (size_t)9 * nchmax * COUT * 16;
    if (smem > 200 * 1024) return EDGE_EINVAL;
    const uint32_t stage = (uint32_t)((smem + 127) / 128 * 128);
    const int nstage = 1;
    const size_t total = (size_t)nstage * stage;
    cudaError_t e = cudaFuncSetAttribute(k_conv_bulk<COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)total);
    if (e != cudaSuccess) return (int)e;
    e = cudaFuncSetAttribute(k_conv_bulk<COUT>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return (int)e;
    const int grid = std::min(g.ntiles, g_sms() * resident_blocks(total, COUT));
    k_conv_bulk<COUT><<<grid, 128, total, st>>>(g, a, b, nin, bias, flags, y, err, nstage, stage);
    return rc_last();
}

template <int CIN>
int launch_wgrad(const Geo& g, const __nv_bfloat16* d, int cout, const __nv_bfloat16* x, float* partial, int nsplit,
                 float* dw, int* err, cudaStream_t st) {
    constexpr int TPG = 9 * CIN <= 512 ? 9 : 3;
    constexpr int NDY = TPG == 9 ? 3 : 1;
    const size_t smem = 8 * 2048 + (size_t)NDY * (CIN / 8) * kSegBytes;
    cudaError_t e = cudaFuncSetAttribute(k_wgrad_tc<CIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    k_wgrad_tc<CIN><<<dim3(27 / TPG, nsplit), 128, smem, st>>>(g, d, cout, x, partial, err);
    int r = rc_last();
    if (r != EDGE_OK) return r;
    k_reduce_wgrad<<<cgrid((long long)cout * CIN * 27), 256, 0, st>>>(partial, nsplit, cout, CIN, dw);
    return rc_last();
}

}  // namespace

extern "C" {

int edge_tc_selftest(int mode, int N, int K, const void* A, const void* B, float* D, int* err, void* stream) {
    if ((mode != 0 && mode != 1) || !A || !B || !D || !err) return EDGE_EINVAL;
    if (N < 16 || N > 256 || N % 16 || K < 16 || K > 256 || K % 16) return EDGE_EINVAL;
    const int M = mode == 0 ? 128 : 64;
    size_t smem = (size_t)(M + N) * K * 2;
    if (smem > 200 * 1024) return EDGE_EINVAL;
    cudaError_t ea = cudaFuncSetAttribute(k_tc_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (ea != cudaSuccess) return (int)ea;
    k_tc_selftest<<<1, 128, smem, (cudaStream_t)stream>>>(mode, N, K, (const __nv_bfloat16*)A,
                                                          (const __nv_bfloat16*)B, D, err);
    return rc_last();
}

int edge_unet_geometry(int X, int Y, int Z, long long* chunk_voxels) {
    if (X < 1 || Y < 1 || Z < 1 || !chunk_voxels) return EDGE_EINVAL;
    Geo g = make_geo(X, Y, Z);
    if ((long long)g.Lc * 8 * 8 >= (1LL << 31)) return EDGE_EINVAL;
    *chunk_voxels = g.Lc;
    return EDGE_OK;
}

int edge_unet_conv(int X, int Y, int Z, const void* x0, const void* w0, int cin0, const void* x1, const void* w1,
                   int cin1, int cout, const float* bias, int flags, void* y, int* err, void* stream) {
    if (!x0 || !w0 || !y || !err || X < 1 || Y < 1 || Z < 1 || (flags & ~3)) return EDGE_EINVAL;
    if (cin0 % 16 || cin0 < 16 || cin0 > 64 || (x1 && (cin1 % 16 || cin1 < 16 || cin1 > 64 || !w1))) return EDGE_EINVAL;
    Geo g = make_geo(X, Y, Z);
    ConvIn a{(const __nv_bfloat16*)x0, (const __nv_bfloat16*)w0, cin0};
    ConvIn b{(const __nv_bfloat16*)x1, (const __nv_bfloat16*)w1, x1 ? cin1 : 0};
    const int nin = x1 ? 2 : 1;
    cudaStream_t st = (cudaStream_t)stream;
    __nv_bfloat16* yo = (__nv_bfloat16*)y;
    switch (cout) {
        case 16: return launch_conv<16>(g, a, b, nin, bias, flags, yo, err, st);
        case 32: return launch_conv<32>(g, a, b, nin, bias, flags, yo, err, st);
        case 64: return launch_conv<64>(g, a, b, nin, bias, flags, yo, err, st);
        default: return EDGE_EINVAL;
    }
}

int edge_unet_wgrad(int X, int Y, int Z, const void* d, int cout, const void* x, int cin, float* partial,
                    int nsplit, float* dw, int* err, void* stream) {
    if (!d || !x || !partial || !dw || !err || nsplit < 1 || cout % 8 || cout < 8 || cout > 64) return EDGE_EINVAL;
    Geo g = make_geo(X, Y, Z);
    cudaStream_t st = (cudaStream_t)stream;
    auto D = (const __nv_bfloat16*)d;
    auto Xp = (const __nv_bfloat16*)x;
    switch (cin) {
        case 16: return launch_wgrad<16>(g, D, cout, Xp, partial, nsplit, dw, err, st);
        case 32: return launch_wgrad<32>(g, D, cout, Xp, partial, nsplit, dw, err, st);
        case 64: return launch_wgrad<64>(g, D, cout, Xp, partial, nsplit, dw, err, st);
        default: return EDGE_EINVAL;
    }
}

int edge_unet_conv_first(int X, int Y, int Z, const float* r, const float* scale, const float* w, const float* bias,
                         void* y, void* stream) {
    if (!r || !scale || !w || !bias || !y) return EDGE_EINVAL;
    Geo g = make_geo(X, Y, Z);
    k_conv_first<<<cgrid((long long)X * Y * Z), 256, 0, (cudaStream_t)stream>>>(g, r, scale, w, bias,
                                                                               (__nv_bfloat16*)y);
    return rc_last();
}

int edge_unet_conv_last(int X, int Y, int Z, const void* f, const float* w, const float* bias, const float* scale,
                        float* z, void* stream) {
    if (!f || !w || !bias || !scale || !z) return EDGE_EINVAL;
    Geo g = make_geo(X, Y, Z);
    k_conv_last<<<cgrid((long long)X * Y * Z), 256, 0, (cudaStream_t)stream>>>(g, (const __nv_bfloat16*)f, w, bias,
                                                                              scale, z);
    return rc_last();
}

int edge_unet_first_bwd(int X, int Y, int Z, const void* d, const float* r, const float* scale, float* partial,
                        int nblk, float* dw, void* stream) {
    if (!d || !r || !scale || !partial || !dw || nblk < 1) return EDGE_EINVAL;
    Geo g = make_geo(X, Y, Z);
    cudaStream_t st = (cudaStream_t)stream;
    k_wgrad_first<<<dim3(27, nblk), 256, 0, st>>>(g, (const __nv_bfloat16*)d, r, scale, partial);
    k_reduce_taps16<<<2, 256, 0, st>>>(partial, nblk, dw);
    return rc_last();
}

int edge_unet_last_bwd(int X, int Y, int Z, const float* dzn, const float* w, const void* f, void* df,
                       float* partial, int nblk, float* dw, void* stream) {
    if (!dzn || !w || !f || !df || !partial || !dw || nblk < 1) return EDGE_EINVAL;
    Geo g = make_geo(X, Y, Z);
    cudaStream_t st = (cudaStream_t)stream;
    k_last_bwd_data<<<cgrid((long long)X * Y * Z), 256, 0, st>>>(g, dzn, w, (__nv_bfloat16*)df);
    k_wgrad_last<<<dim3(27, nblk), 256, 0, st>>>(g, dzn, (const __nv_bfloat16*)f, partial);
    k_reduce_taps16<<<2, 256, 0, st>>>(partial, nblk, dw);
    return rc_last();
}

int edge_unet_chan_sum(int X, int Y, int Z, int channels, const void* d, float* partial, int nblk, float* out,
                       void* stream) {
    if (!d || !partial || !out || channels % 8 || nblk < 1) return EDGE_EINVAL;
    Geo g = make_geo(X, Y, Z);
    cudaStream_t st = (cudaStream_t)stream;
    k_chan_sum<<<dim3(channels / 8, nblk), 256, 0, st>>>(g.Lc, (const __nv_bfloat16*)d, partial);
    k_reduce_chan<<<1, 64, 0, st>>>(partial, nblk, channels, out);
    return rc_last();
}

int edge_unet_relu_bwd(int X, int Y, int Z, int channels, const void* dy, const void* y, void* out, void* stream) {
    if (!dy || !y || !out || channels % 8) return EDGE_EINVAL;
    Geo g = make_geo(X, Y, Z);
    const long long n8 = (long long)(channels / 8) * g.Lc;
    k_relu_bwd<<<cgrid(n8), 256, 0, (cudaStream_t)stream>>>(n8, (const __nv_bfloat16*)dy, (const __nv_bfloat16*)y,
                                                           (__nv_bfloat16*)out);
    return rc_last();
}

int edge_unet_pool(int X, int Y, int Z, int channels, const void* fine, void* coarse, void* stream) {
    if (!fine || !coarse || X % 2 || Y % 2 || Z % 2 || channels % 8) return EDGE_EINVAL;
    Geo gf = make_geo(X, Y, Z), gc = make_geo(X / 2, Y / 2, Z / 2);
    k_pool<<<cgrid((long long)X * Y * Z / 8 * (channels / 8)), 256, 0, (cudaStream_t)stream>>>(
        gf, gc, channels / 8, (const __nv_bfloat16*)fine, (__nv_bfloat16*)coarse);
    return rc_last();
}

int edge_unet_pool_bwd(int X, int Y, int Z, int channels, const void* dcoarse, void* dfine, int accum, void* stream) {
    if (!dfine || !dcoarse || X % 2 || Y % 2 || Z % 2 || channels % 8) return EDGE_EINVAL;
    Geo gf = make_geo(X, Y, Z), gc = make_geo(X / 2, Y / 2, Z / 2);
    k_pool_bwd<<<cgrid((long long)X * Y * Z * (channels / 8)), 256, 0, (cudaStream_t)stream>>>(
        gf, gc, channels / 8, (const __nv_bfloat16*)dcoarse, (__nv_bfloat16*)dfine, accum);
    return rc_last();
}

int edge_unet_upsample(int X, int Y, int Z, int channels, const void* coarse, void* fine, void* stream) {
    if (!fine || !coarse || X % 2 || Y % 2 || Z % 2 || channels % 8) return EDGE_EINVAL;
    Geo gf = make_geo(X, Y, Z), gc = make_geo(X / 2, Y / 2, Z / 2);
    k_upsample<<<cgrid((long long)X * Y * Z * (channels / 8)), 256, 0, (cudaStream_t)stream>>>(
        gc, gf, channels / 8, (const __nv_bfloat16*)coarse, (__nv_bfloat16*)fine);
    return rc_last();
}

int edge_unet_up_bwd(int X, int Y, int Z, int channels, const void* dfine, void* dcoarse, void* stream) {
    if (!dfine || !dcoarse || X % 2 || Y % 2 || Z % 2 || channels % 8) return EDGE_EINVAL;
    Geo gf = make_geo(X, Y, Z), gc = make_geo(X / 2, Y / 2, Z / 2);
    k_up_bwd<<<cgrid((long long)X * Y * Z / 8 * (channels / 8)), 256, 0, (cudaStream_t)stream>>>(
        gc, gf, channels / 8, (const __nv_bfloat16*)dfine, (__nv_bfloat16*)dcoarse);
    return rc_last();
}

int edge_unet_pack_weights(const float* w, int cout, int cin, int transpose, void* out, void* stream) {
    if (!w || !out || cout % 8 || cin % 8) return EDGE_EINVAL;
    k_pack_weights<<<cgrid((long long)cout * cin * 27), 256, 0, (cudaStream_t)stream>>>(w, cout, cin, transpose,
                                                                                       (__nv_bfloat16*)out);
    return rc_last();
}

int edge_unet_input_scale(const float* r, long long n, void* work, float* scale, void* stream) {
    if (!r || !scale || !work || n <= 0) return EDGE_EINVAL;
    // work: 1024 doubles of partial sums, then the arrival counter (zero on entry, reset on exit)
    double* partial = (double*)work;
    unsigned* counter = (unsigned*)(partial + 1024);
    const int grid = (int)std::min<long long>(1024, std::max<long long>(1, (n + 255) / 256));
    k_input_scale<<<grid, 256, 0, (cudaStream_t)stream>>>(r, n, partial, counter, scale);
    return rc_last();
}

int edge_unet_loss(const float* z, const float* target, const float* scale, long long n, double* stats, float* dzn,
                   void* stream) {
    if (!z || !target || !scale || !stats || !dzn || n <= 0) return EDGE_EINVAL;
    cudaStream_t st = (cudaStream_t)stream;
    k_loss_stats<<<1, 1024, 0, st>>>(z, target, scale, n, stats);
    k_loss_grad<<<cgrid(n), 256, 0, st>>>(z, target, scale, stats, n, dzn);
    return rc_last();
}

int edge_unet_adam(long long n, float* p, const float* g, float* m, float* v, float lr, float b1, float b2, float eps,
                   int step, void* stream) {
    if (!p || !g || !m || !v || n <= 0 || step < 1) return EDGE_EINVAL;
    const float bc1 = 1.0f - powf(b1, (float)step), bc2 = 1.0f - powf(b2, (float)step);
    k_adam<<<cgrid(n), 256, 0, (cudaStream_t)stream>>>(n, p, g, m, v, lr, b1, b2, eps, bc1, bc2);
    return rc_last();
}

}  // extern "C"
