// Device code of the voxel solve (sm_100a). Included by solver.cu only.
//
// Data layout in HBM, per level: xyz-interleaved DOF vectors (DOF 3n + d, node n = i + NX (j + NY k),
// the reference's layout), one 32-bit word per voxel (0 empty, float bits of s for s * Kb,
// OWN_BIT | index of an own 24x24 matrix), one mask byte per node (fixed DOFs, active, uniform).
// The level's Kb (576) and its assembled 27-point stencil (243) travel as kernel parameters, so
// every coefficient is a constant-bank operand of the FMA that uses it.
#pragma once

#include <cuda_fp16.h>
#include <cstdint>

namespace psfea {
namespace dev {

constexpr uint32_t OWN_BIT = 0x80000000u;
constexpr uint8_t NM_ACTIVE = 8, NM_UNIFORM = 16;

struct LevelView {
    int nx, ny, nz, NX, NY, NZ;
    long long nNodes;
    const uint32_t* word;
    const uint8_t* nmask;
    const float* own;       // own matrices, 32-bit
    const __half* own16;    // the same as halves times hs (mixed precision), or null
    float hs;
    const double* dadd;     // diagonal shift per DOF, or null
    const float* dadd32;
    const float* invD;      // 1 / diag per DOF (0 where fixed), 32-bit
};

template <class T>
struct Coefs {
    T S[243];   // [m][3 d + c], m = (ox+1) + 3 (oy+1) + 9 (oz+1)
    T Kb[576];  // row-major 24x24
};

// corner index of the unit offset (x, y, z)
__host__ __device__ constexpr int cornerOf(int x, int y, int z) { return (y ? (x ? 2 : 3) : (x ? 1 : 0)) + 4 * z; }

// (K x) at node (i, j, k). Uniform nodes: s times the assembled stencil, structural zeros skipped
// (entry (d, c) of neighbour o is zero by the cube's reflection symmetry unless d == c or both
// o_d and o_c are nonzero: 153 of 243). Others: the rows of the node's corner in each of its up
// to 8 voxels (native/src/fea/voxel_fea.cpp:422-486 computes the same sums).
//
// DIFF: every value enters as its difference from the node's own value, x_m - x_n. Rows of K
// annihilate rigid translations, so the product is unchanged in exact arithmetic, but its 32-bit
// rounding error then scales with the field's local variation instead of its magnitude: what keeps
// the FP32 CG accurate on smooth search directions. (The reference's WGSL kernel forms its
// products the same way, native/shaders/fea.wgsl:91-92.) The diagonal shift is not a
// translation-free term and always uses x_n itself.
template <class T, bool OWN16, bool DIFF = false>
__device__ __forceinline__ void applyAt(const LevelView& L, const Coefs<T>& C, const T* __restrict__ x, int i, int j, int k,
                                        long long n, uint8_t mask, T acc[3]) {
    acc[0] = acc[1] = acc[2] = T(0);
    if (!(mask & NM_ACTIVE)) return;
    const long long NX = L.NX, NXY = (long long)L.NX * L.NY;
    T own0 = 0, own1 = 0, own2 = 0;
    if (DIFF) {
        own0 = __ldg(x + 3 * n);
        own1 = __ldg(x + 3 * n + 1);
        own2 = __ldg(x + 3 * n + 2);
    }
    if (mask & NM_UNIFORM) {
        const float s = __uint_as_float(__ldg(L.word + ((i - 1) + (long long)L.nx * ((j - 1) + (long long)L.ny * (k - 1)))));
        T a0 = 0, a1 = 0, a2 = 0;
#pragma unroll
        for (int m = 0; m < 27; m++) {
            const int ox = m % 3 - 1, oy = (m / 3) % 3 - 1, oz = m / 9 - 1;
            if (DIFF && m == 13) continue;  // the node itself: a zero difference
            const T* xp = x + 3 * (n + ox + oy * NX + oz * NXY);
            const T x0 = __ldg(xp) - own0, x1 = __ldg(xp + 1) - own1, x2 = __ldg(xp + 2) - own2;
            a0 += C.S[m * 9 + 0] * x0;
            a1 += C.S[m * 9 + 4] * x1;
            a2 += C.S[m * 9 + 8] * x2;
            if (ox && oy) { a0 += C.S[m * 9 + 1] * x1; a1 += C.S[m * 9 + 3] * x0; }
            if (ox && oz) { a0 += C.S[m * 9 + 2] * x2; a2 += C.S[m * 9 + 6] * x0; }
            if (oy && oz) { a1 += C.S[m * 9 + 5] * x2; a2 += C.S[m * 9 + 7] * x1; }
        }
        acc[0] = T(s) * a0;
        acc[1] = T(s) * a1;
        acc[2] = T(s) * a2;
    } else {
#pragma unroll
        for (int v = 0; v < 8; v++) {
            const int di = v & 1, dj = (v >> 1) & 1, dk = v >> 2;
            const int ei = i - 1 + di, ej = j - 1 + dj, ek = k - 1 + dk;
            if (ei < 0 || ej < 0 || ek < 0 || ei >= L.nx || ej >= L.ny || ek >= L.nz) continue;
            const uint32_t w = __ldg(L.word + (ei + (long long)L.nx * (ej + (long long)L.ny * ek)));
            if (w == 0) continue;
            const int a = cornerOf(1 - di, 1 - dj, 1 - dk);
            // the voxel's 8 corner values
            T xe[24];
#pragma unroll
            for (int b = 0; b < 8; b++) {
                const int bx = (b == 1 || b == 2 || b == 5 || b == 6), by = (b == 2 || b == 3 || b == 6 || b == 7), bz = b >> 2;
                const T* xp = x + 3 * (n + (di + bx - 1) + (dj + by - 1) * NX + (dk + bz - 1) * NXY);
                xe[3 * b] = __ldg(xp) - own0;
                xe[3 * b + 1] = __ldg(xp + 1) - own1;
                xe[3 * b + 2] = __ldg(xp + 2) - own2;
            }
            if (!(w & OWN_BIT)) {
                T t0 = 0, t1 = 0, t2 = 0;
#pragma unroll
                for (int q = 0; q < 24; q++) {
                    t0 += C.Kb[(3 * a + 0) * 24 + q] * xe[q];
                    t1 += C.Kb[(3 * a + 1) * 24 + q] * xe[q];
                    t2 += C.Kb[(3 * a + 2) * 24 + q] * xe[q];
                }
                const T s = T(__uint_as_float(w));
                acc[0] += s * t0;
                acc[1] += s * t1;
                acc[2] += s * t2;
            } else if (OWN16) {
                const __half2* K2 = reinterpret_cast<const __half2*>(L.own16 + (long long)(w & ~OWN_BIT) * 576 + 72 * a);
                T t[3] = {0, 0, 0};
#pragma unroll
                for (int d = 0; d < 3; d++)
#pragma unroll
                    for (int q = 0; q < 12; q++) {
                        const float2 kv = __half22float2(__ldg(K2 + d * 12 + q));
                        t[d] += T(kv.x) * xe[2 * q] + T(kv.y) * xe[2 * q + 1];
                    }
                acc[0] += T(L.hs) * t[0];
                acc[1] += T(L.hs) * t[1];
                acc[2] += T(L.hs) * t[2];
            } else {
                const float4* K4 = reinterpret_cast<const float4*>(L.own + (long long)(w & ~OWN_BIT) * 576 + 72 * a);
#pragma unroll
                for (int d = 0; d < 3; d++)
#pragma unroll
                    for (int q = 0; q < 6; q++) {
                        const float4 kv = __ldg(K4 + d * 6 + q);
                        acc[d] += T(kv.x) * xe[4 * q] + T(kv.y) * xe[4 * q + 1] + T(kv.z) * xe[4 * q + 2] + T(kv.w) * xe[4 * q + 3];
                    }
            }
        }
    }
    if (L.dadd) {
#pragma unroll
        for (int d = 0; d < 3; d++) acc[d] += (sizeof(T) == 8 ? T(L.dadd[3 * n + d]) : T(L.dadd32[3 * n + d])) * x[3 * n + d];
    }
}

__device__ __forceinline__ void nodeCoords(const LevelView& L, long long n, int& i, int& j, int& k) {
    const long long row = n / L.NX;
    i = int(n - row * L.NX);
    j = int(row % L.NY);
    k = int(row / L.NY);
}

// ---- deterministic grid reductions: per-block tree sums, the last block folds the partials in
// block order (so results are bitwise reproducible for a given launch shape) ----

template <int K>
__device__ __forceinline__ void warpReduce(double (&v)[K], unsigned maxMask) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int q = 0; q < K; q++) {
            const double w = __shfl_down_sync(0xffffffffu, v[q], o);
            v[q] = ((maxMask >> q) & 1) ? fmax(v[q], w) : v[q] + w;
        }
}

// Reduces v over the block into out (thread 0's copy valid). sh: 32 * K doubles of shared memory.
template <int K>
__device__ __forceinline__ void blockReduce(double (&v)[K], unsigned maxMask, double* sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    warpReduce<K>(v, maxMask);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < K; q++) sh[wid * K + q] = v[q];
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int q = 0; q < K; q++) v[q] = lane < nw ? sh[lane * K + q] : 0.0;
        warpReduce<K>(v, maxMask);
    }
}

// Whole-grid reduction: every block writes its partial; returns true in the last block to finish,
// where out[] (in every thread) holds the totals. ticket must start at 0 and is left at 0.
template <int K>
__device__ bool gridReduce(double (&v)[K], unsigned maxMask, double* partials, unsigned* ticket, double (&out)[K]) {
    __shared__ double sh[32 * K];
    __shared__ bool last;
    blockReduce<K>(v, maxMask, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < K; q++) partials[(size_t)blockIdx.x * K + q] = v[q];
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double acc[K];
#pragma unroll
    for (int q = 0; q < K; q++) acc[q] = 0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
        for (int q = 0; q < K; q++) {
            const double p = __ldcg(partials + (size_t)b * K + q);
            acc[q] = ((maxMask >> q) & 1) ? fmax(acc[q], p) : acc[q] + p;
        }
    __syncthreads();
    blockReduce<K>(acc, maxMask, sh);
    __shared__ double res[K];
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < K; q++) res[q] = acc[q];
        *ticket = 0;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < K; q++) out[q] = res[q];
    return true;
}

}  // namespace dev
}  // namespace psfea
