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

namespace psfea {
namespace dev {

// ---------------------------------------------------------------- tiled operator
//
// One CTA per 32 x 8 x 8 node tile (only tiles with an active node are launched). The CTA stages
// the tile's x values with a one-node halo (34 x 10 x 10 nodes) and the voxel words around it
// (33 x 9 x 9) in shared memory with one burst of coalesced loads, all in flight together, then
// computes its 2048 nodes from shared memory: uniform nodes with the 153-FMA assembled stencil,
// the other active nodes (compacted in a fixed order) with the per-voxel gather, so the two code
// paths never share a warp. Inactive nodes of the tile are written 0; inactive tiles are never
// touched (their outputs are 0 already).

constexpr int TX = 32, TY = 8, TZ = 4, TILE_THREADS = TX * TY, TILE_NODES = TX * TY * TZ;
constexpr int HX = TX + 2, HY = TY + 2, HZ = TZ + 2, PROW = 3 * HX;  // x with halo; values per row
constexpr int VX = TX + 1, VY = TY + 1, VZ = TZ + 1;                 // voxel words with halo

enum { TOP_APPLY = 0, TOP_CHEB = 1, TOP_RESID = 2, TOP_DOT = 3 };

template <class T>
struct TileIO {
    const T* x;        // input vector
    T* y;              // output vector
    const float* r;    // CHEB / RESID: right-hand side (32-bit level vectors)
    float* d;          // CHEB: Chebyshev direction, updated in place
    float c1, c2;      // CHEB: d = c1 d + c2 D^-1 (r - K x)
    int raw;           // APPLY: keep held DOFs
};

__host__ __device__ constexpr uint32_t packTile(int tx, int ty, int tz) { return uint32_t(tx) | (uint32_t(ty) << 11) | (uint32_t(tz) << 22); }

// x halo, voxel words, per-node K x results (row-major like the global tile rows), node masks,
// the gather list and the warp counts
// every part starts on a 16-byte boundary
__host__ __device__ constexpr size_t align16(size_t b) { return (b + 15) & ~size_t(15); }
template <class T> __host__ __device__ constexpr size_t tileOffV() { return align16(sizeof(T) * HZ * HY * PROW); }
template <class T> __host__ __device__ constexpr size_t tileOffK() { return tileOffV<T>() + align16(sizeof(uint32_t) * VZ * VY * VX); }
template <class T> __host__ __device__ constexpr size_t tileOffM() { return tileOffK<T>() + align16(sizeof(T) * 3 * TILE_NODES); }
template <class T> __host__ __device__ constexpr size_t tileOffB() { return tileOffM<T>() + align16(TILE_NODES); }
template <class T> __host__ __device__ constexpr size_t tileSmemBytes() { return tileOffB<T>() + sizeof(int) * (TILE_NODES + 32); }

// asynchronous global -> shared copy of one 4- or 8-byte element, zero-filled when !valid
template <int BYTES>
__device__ __forceinline__ void cpAsync(void* dst, const void* src, bool valid) {
    const unsigned d = unsigned(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(d), "l"(src), "n"(BYTES), "r"(valid ? BYTES : 0) : "memory");
}
__device__ __forceinline__ void cpAsyncWaitAll() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// shared-memory offsets of x value (node tx + ox, ty + oy, tz + oz of the tile, component 0) and of
// the voxel word at tile voxel (vx, vy, vz) (both with the halo offset of one)
__device__ __forceinline__ int xOff(int cx, int cy, int cz) { return ((cz + 1) * HY + (cy + 1)) * PROW + 3 * (cx + 1); }
__device__ __forceinline__ int vOff(int vx, int vy, int vz) { return (vz * VY + vy) * VX + vx; }

template <class T, bool OWN16, bool DIFF>
struct TileOp {
    // K x at tile node (cx, cy, cz) by the per-voxel gather; own = the node's value when DIFF
    static __device__ __forceinline__ void general(const LevelView& L, const Coefs<T>& C, const T* xs, const uint32_t* vs, int cx, int cy,
                                                   int cz, T acc[3], const T own[3]) {
        acc[0] = acc[1] = acc[2] = T(0);
#pragma unroll
        for (int v = 0; v < 8; v++) {
            const int di = v & 1, dj = (v >> 1) & 1, dk = v >> 2;
            // voxel (i - 1 + di, ...) is tile voxel (cx + di, cy + dj, cz + dk) with the halo offset
            const uint32_t w = vs[vOff(cx + di, cy + dj, cz + dk)];
            if (w == 0) continue;
            const int a = cornerOf(1 - di, 1 - dj, 1 - dk);
            T xe[24];
#pragma unroll
            for (int b = 0; b < 8; b++) {
                const int bx = (b == 1 || b == 2 || b == 5 || b == 6), by = (b == 2 || b == 3 || b == 6 || b == 7), bz = b >> 2;
                const T* xp = xs + xOff(cx + di + bx - 1, cy + dj + by - 1, cz + dk + bz - 1);
                xe[3 * b] = xp[0] - own[0];
                xe[3 * b + 1] = xp[1] - own[1];
                xe[3 * b + 2] = xp[2] - own[2];
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

    // unscaled stencil sums of the thread's whole column (cz = 0..TZ-1) at once: every plane of the
    // 3x3 neighbourhood is read from shared memory once and feeds the (up to) three column nodes it
    // neighbours. With DIFF every value enters as its difference from the output node's own value.
    static __device__ __forceinline__ void column(const Coefs<T>& C, const T* xs, int cx, int cy, T acc[TZ][3]) {
#pragma unroll
        for (int z = 0; z < TZ; z++) acc[z][0] = acc[z][1] = acc[z][2] = T(0);
        T own[TZ][3];
#pragma unroll
        for (int z = 0; z < TZ; z++) {
            const T* xr = xs + xOff(cx, cy, z);
            own[z][0] = DIFF ? xr[0] : T(0);
            own[z][1] = DIFF ? xr[1] : T(0);
            own[z][2] = DIFF ? xr[2] : T(0);
        }
#pragma unroll
        for (int p = -1; p <= TZ; p++) {
            T v[9][3];
#pragma unroll
            for (int b = 0; b < 9; b++) {
                const T* xp = xs + xOff(cx + b % 3 - 1, cy + b / 3 - 1, p);
                v[b][0] = xp[0];
                v[b][1] = xp[1];
                v[b][2] = xp[2];
            }
#pragma unroll
            for (int z = p - 1; z <= p + 1; z++) {
                if (z < 0 || z >= TZ) continue;
                const int oz = p - z;
#pragma unroll
                for (int b = 0; b < 9; b++) {
                    const int ox = b % 3 - 1, oy = b / 3 - 1, m = (ox + 1) + 3 * (oy + 1) + 9 * (oz + 1);
                    if (DIFF && m == 13) continue;  // the node itself: a zero difference
                    const T x0 = v[b][0] - own[z][0], x1 = v[b][1] - own[z][1], x2 = v[b][2] - own[z][2];
                    T* a = acc[z];
                    a[0] += C.S[m * 9 + 0] * x0;
                    a[1] += C.S[m * 9 + 4] * x1;
                    a[2] += C.S[m * 9 + 8] * x2;
                    if (ox && oy) { a[0] += C.S[m * 9 + 1] * x1; a[1] += C.S[m * 9 + 3] * x0; }
                    if (ox && oz) { a[0] += C.S[m * 9 + 2] * x2; a[2] += C.S[m * 9 + 6] * x0; }
                    if (oy && oz) { a[1] += C.S[m * 9 + 5] * x2; a[2] += C.S[m * 9 + 7] * x1; }
                }
            }
        }
    }

    // s * (assembled stencil . x) at tile node (cx, cy, cz)
    static __device__ __forceinline__ void stencil(const Coefs<T>& C, const T* xs, int cx, int cy, int cz, float s, T acc[3], const T own[3]) {
        T a0 = 0, a1 = 0, a2 = 0;
#pragma unroll
        for (int m = 0; m < 27; m++) {
            const int ox = m % 3 - 1, oy = (m / 3) % 3 - 1, oz = m / 9 - 1;
            if (DIFF && m == 13) continue;
            const T* xp = xs + xOff(cx + ox, cy + oy, cz + oz);
            const T x0 = xp[0] - own[0], x1 = xp[1] - own[1], x2 = xp[2] - own[2];
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
    }
};

}  // namespace dev
}  // namespace psfea
