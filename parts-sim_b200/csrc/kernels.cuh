// Device code of the voxel solve (sm_100a). Included by solver.cu only.
//
// Data layout in HBM, per level: xyz-interleaved DOF vectors (DOF 3n + d) over pitched node rows,
// node n = i + PX (j + NY k) with the row pitch PX = NX rounded up to a multiple of 4, so that every
// row of 3 PX values starts on a 16-byte boundary (the rule of tensor-memory-access copies); the
// padding nodes i >= NX are inactive with all DOFs held, and stay 0 in every vector. One 32-bit word
// per voxel (0 empty, float bits of s for s * Kb, OWN_BIT | index of an own 24x24 matrix) over rows
// of px = nx rounded up to a multiple of 4 words (padding words 0), one mask byte per node (fixed
// DOFs, active, uniform). The reference's dense layout (pitch NX) exists only at the C ABI.
// The level's Kb (576) and its assembled 27-point stencil (243) travel as kernel parameters, so
// every coefficient is a constant-bank operand of the FMA that uses it.
#pragma once

#include <cuda.h>
#include <cuda_fp16.h>
#include <cstdint>

namespace psfea {
namespace dev {

constexpr uint32_t OWN_BIT = 0x80000000u;
constexpr uint8_t NM_ACTIVE = 8, NM_UNIFORM = 16;

struct LevelView {
    int nx, ny, nz, NX, NY, NZ;  // voxel and node counts per axis
    int PX, px;                  // row pitches: nodes (PX >= NX) and voxel words (px >= nx), multiples of 4
    long long nNodes;            // PX NY NZ: the length of every per-node array
    const uint32_t* word;
    const uint8_t* nmask;
    const float* own;       // own matrices, 32-bit
    const __half* own16;    // the same as halves times hs (mixed precision), or null
    float hs;
    const double* dadd;     // diagonal shift per DOF, or null
    const float* dadd32;
    const float* invD;      // 1 / diag per DOF (0 where fixed), 32-bit
    __host__ __device__ long long wi(int i, int j, int k) const { return i + (long long)px * (j + (long long)ny * k); }
};

template <class T>
struct Coefs {
    alignas(16) T Kb[576];  // row-major 24x24 (16-byte aligned: read as pairs by the paired FMAs)
    T S[243];               // [m][3 d + c], m = (ox+1) + 3 (oy+1) + 9 (oz+1)
};
// the 32-bit coefficients also as duplicated pairs (s, s), the operand of a paired FMA that
// advances two nodes at once
struct Coefs32 : Coefs<float> {
    float2 S2[243];
};

// corner index of the unit offset (x, y, z)
__host__ __device__ constexpr int cornerOf(int x, int y, int z) { return (y ? (x ? 2 : 3) : (x ? 1 : 0)) + 4 * z; }

// the three rows of corner a of a 24x24 matrix times the 24 corner values xe, added to t[3]:
//   Kb (the level's uniform matrix, kernel parameter): 32-bit values pair consecutive columns in
//   paired FMAs (__ffma2_rn; the pair's two partial sums are added at the end)
//   own16 (FP16 Galerkin matrices): 16-byte loads of eight halves each, widened to the value type
template <class T>
__device__ __forceinline__ void kbRows(const T* Kb, int a, const T xe[24], T t[3]) {
    if constexpr (sizeof(T) == 4) {
        const float2* K2 = reinterpret_cast<const float2*>(Kb) + 36 * a;
        float2 p0 = make_float2(0.f, 0.f), p1 = p0, p2 = p0;
#pragma unroll
        for (int q = 0; q < 12; q++) {
            const float2 xq = make_float2(xe[2 * q], xe[2 * q + 1]);
            p0 = __ffma2_rn(K2[q], xq, p0);
            p1 = __ffma2_rn(K2[12 + q], xq, p1);
            p2 = __ffma2_rn(K2[24 + q], xq, p2);
        }
        t[0] = p0.x + p0.y;
        t[1] = p1.x + p1.y;
        t[2] = p2.x + p2.y;
    } else {
        T t0 = 0, t1 = 0, t2 = 0;
#pragma unroll
        for (int q = 0; q < 24; q++) {
            t0 += Kb[(3 * a + 0) * 24 + q] * xe[q];
            t1 += Kb[(3 * a + 1) * 24 + q] * xe[q];
            t2 += Kb[(3 * a + 2) * 24 + q] * xe[q];
        }
        t[0] = t0;
        t[1] = t1;
        t[2] = t2;
    }
}
// SMEM: M is in shared memory (plain loads; the read-only global path otherwise)
template <class T, bool SMEM = false>
__device__ __forceinline__ void own16Rows(const __half* M, const T xe[24], T t[3]) {
    const uint4* K16 = reinterpret_cast<const uint4*>(M);  // 72 halves: rows d at [24 d, 24 d + 24)
#pragma unroll
    for (int d = 0; d < 3; d++) {
        T acc = 0;
#pragma unroll
        for (int g = 0; g < 3; g++) {
            const uint4 u = SMEM ? K16[3 * d + g] : __ldg(K16 + 3 * d + g);
            const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const float2 kv = __half22float2(*reinterpret_cast<const __half2*>(&w[e]));
                acc += T(kv.x) * xe[8 * g + 2 * e] + T(kv.y) * xe[8 * g + 2 * e + 1];
            }
        }
        t[d] = acc;
    }
}

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
//
// x is read at node index n with row pitch XP (L.PX for the level's own vectors); the diagonal
// shift at the level's node index nm. S: the stride between consecutive DOFs of x (1 for one
// vector; the block width for the RHS-minor layout of a multi-RHS block, x then pointing at the
// lane's right-hand side). SMEM: L.own / L.own16 point at a copy in shared memory.
template <class T, bool OWN16, bool DIFF = false, int S = 1, bool SMEM = false>
__device__ __forceinline__ void applyAt(const LevelView& L, const Coefs<T>& C, const T* __restrict__ x, int i, int j, int k,
                                        long long n, uint8_t mask, T acc[3], long long XP, long long nm) {
    acc[0] = acc[1] = acc[2] = T(0);
    if (!(mask & NM_ACTIVE)) return;
    const long long NX = XP, NXY = XP * L.NY;
    T own0 = 0, own1 = 0, own2 = 0;
    if (DIFF) {
        own0 = __ldg(x + 3 * S * n);
        own1 = __ldg(x + 3 * S * n + S);
        own2 = __ldg(x + 3 * S * n + 2 * S);
    }
    if (mask & NM_UNIFORM) {
        const float s = __uint_as_float(__ldg(L.word + L.wi(i - 1, j - 1, k - 1)));
        T a0 = 0, a1 = 0, a2 = 0;
#pragma unroll
        for (int m = 0; m < 27; m++) {
            const int ox = m % 3 - 1, oy = (m / 3) % 3 - 1, oz = m / 9 - 1;
            if (DIFF && m == 13) continue;  // the node itself: a zero difference
            const T* xp = x + 3 * S * (n + ox + oy * NX + oz * NXY);
            const T x0 = __ldg(xp) - own0, x1 = __ldg(xp + S) - own1, x2 = __ldg(xp + 2 * S) - own2;
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
            const uint32_t w = __ldg(L.word + L.wi(ei, ej, ek));
            if (w == 0) continue;
            const int a = cornerOf(1 - di, 1 - dj, 1 - dk);
            // the voxel's 8 corner values
            T xe[24];
#pragma unroll
            for (int b = 0; b < 8; b++) {
                const int bx = (b == 1 || b == 2 || b == 5 || b == 6), by = (b == 2 || b == 3 || b == 6 || b == 7), bz = b >> 2;
                const T* xp = x + 3 * S * (n + (di + bx - 1) + (dj + by - 1) * NX + (dk + bz - 1) * NXY);
                xe[3 * b] = __ldg(xp) - own0;
                xe[3 * b + 1] = __ldg(xp + S) - own1;
                xe[3 * b + 2] = __ldg(xp + 2 * S) - own2;
            }
            if (!(w & OWN_BIT)) {
                T t[3];
                kbRows<T>(C.Kb, a, xe, t);
                const T s = T(__uint_as_float(w));
                acc[0] += s * t[0];
                acc[1] += s * t[1];
                acc[2] += s * t[2];
            } else if (OWN16) {
                T t[3];
                own16Rows<T, SMEM>(L.own16 + (long long)(w & ~OWN_BIT) * 576 + 72 * a, xe, t);
                acc[0] += T(L.hs) * t[0];
                acc[1] += T(L.hs) * t[1];
                acc[2] += T(L.hs) * t[2];
            } else {
                const float4* K4 = reinterpret_cast<const float4*>(L.own + (long long)(w & ~OWN_BIT) * 576 + 72 * a);
#pragma unroll
                for (int d = 0; d < 3; d++)
#pragma unroll
                    for (int q = 0; q < 6; q++) {
                        const float4 kv = SMEM ? K4[d * 6 + q] : __ldg(K4 + d * 6 + q);
                        acc[d] += T(kv.x) * xe[4 * q] + T(kv.y) * xe[4 * q + 1] + T(kv.z) * xe[4 * q + 2] + T(kv.w) * xe[4 * q + 3];
                    }
            }
        }
    }
    if (L.dadd) {
#pragma unroll
        for (int d = 0; d < 3; d++) acc[d] += (sizeof(T) == 8 ? T(L.dadd[3 * nm + d]) : T(L.dadd32[3 * nm + d])) * x[(3 * n + d) * S];
    }
}

// a read-only vector entry as T: FP32 / FP64 storage as is, FP16 storage converted
template <class T>
__device__ __forceinline__ T ldv(const float* p) { return T(__ldg(p)); }
template <class T>
__device__ __forceinline__ T ldv(const double* p) { return T(__ldg(p)); }
template <class T>
__device__ __forceinline__ T ldv(const __half* p) { return T(__half2float(__ldg(p))); }
__device__ __forceinline__ void stv(float* p, float v) { *p = v; }
__device__ __forceinline__ void stv(__half* p, float v) { *p = __float2half_rn(v); }
__device__ __forceinline__ float ldf(const float* p) { return *p; }
__device__ __forceinline__ float ldf(const __half* p) { return __half2float(*p); }

// Layout: coefficient c = 9 m + 3 p + q (m the neighbour (ox + 1) + 3 (oy + 1) + 9 (oz + 1), p the
// row and q the column component) of listed node t sits in chunk c / CW of CW consecutive values
// (16 bytes: CW = 4 floats or 8 halves), chunks stored chunk-major over the nodes, so that a warp
// reads one chunk of 32 consecutive nodes as 512 contiguous bytes. The tail of the last chunk is 0.
template <int CW>
__host__ __device__ constexpr int stnChunks() { return (243 + CW - 1) / CW; }
template <int CW>
__host__ __device__ __forceinline__ long long stnAt(int c, long long t, long long count) { return ((c / CW) * count + t) * CW + c % CW; }

// one 16-byte chunk of coefficients as floats
__device__ __forceinline__ void ldChunk(const float* p, float (&v)[4]) {
    const float4 u = __ldcs(reinterpret_cast<const float4*>(p));
    v[0] = u.x;
    v[1] = u.y;
    v[2] = u.z;
    v[3] = u.w;
}
__device__ __forceinline__ void ldChunk(const __half* p, float (&v)[8]) {
    const uint4 u = __ldcs(reinterpret_cast<const uint4*>(p));
    const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
    for (int e = 0; e < 4; e++) {
        const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&w[e]));
        v[2 * e] = f.x;
        v[2 * e + 1] = f.y;
    }
}

__device__ __forceinline__ void ldChunk(const double* p, double (&v)[2]) {
    const double2 u = __ldcs(reinterpret_cast<const double2*>(p));
    v[0] = u.x;
    v[1] = u.y;
}

__device__ __forceinline__ void nodeCoords(const LevelView& L, long long n, int& i, int& j, int& k) {
    if (n <= 0xffffffffLL) {  // two 32-bit divisions: a 64-bit one is a long software sequence
        const unsigned u = unsigned(n), px = unsigned(L.PX), ny = unsigned(L.NY);
        const unsigned row = u / px, kk = row / ny;
        i = int(u - row * px);
        j = int(row - kk * ny);
        k = int(kk);
        return;
    }
    const long long row = n / L.PX;
    i = int(n - row * L.PX);
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
// One CTA per 32 x 8 x 4 node tile (only tiles with an active node are launched). One thread stages
// what the tile needs with tensor-memory-access (TMA) copies on two shared-memory barriers: the x
// values with a one-node halo and the voxel words around the tile first, the tile's r and d (the
// smoother and residual epilogues) second. Each thread then computes its column of four nodes with
// the 153-FMA assembled stencil from shared memory (uniform nodes) and runs their epilogues in
// shared memory. Boundary nodes (active, not uniform): 32-bit tiles compact them in a fixed order
// and give one thread each the per-voxel gather, packed into as few warps as possible; 64-bit tiles
// leave them to the boundary-node kernel that follows, which overwrites their output slots (the
// FP64 gather is heavy enough to want a launch of its own at full occupancy). One thread writes
// the tile back with TMA stores. Inactive nodes are written 0; inactive tiles are never touched
// (their outputs are 0 already).
//
// TMA boxes start on 16-byte boundaries: node rows are pitched (PX, a multiple of 4) and the halo
// box starts 4 nodes (12 values) left of the tile instead of 1, the voxel box 4 words left of it;
// boxes reaching outside the grid read zeros.

constexpr int TX = 32, TY = 8, TZ = 4, TILE_THREADS = TX * TY, TILE_NODES = TX * TY * TZ;
constexpr int HY = TY + 2, HZ = TZ + 2;          // x halo rows and planes
constexpr int XLEFT = 4;                         // halo box starts XLEFT nodes left of the tile
// halo box row: nodes i0-4 .. i0+33 (111 values) padded to 116, so that the plane stride of the
// shared-memory halo (10 rows, 1160 words) is not a multiple of the 32 banks: the four planes of a
// column then sit in different banks when the lanes of a warp take the nodes of a few columns
constexpr int PROW = 116;
constexpr int VX = TX + 1, VY = TY + 1, VZ = TZ + 1;  // voxel words needed per axis
constexpr int WROW = 36;                         // voxel box row: words i0-4 .. i0+31 (144 bytes)
constexpr int TROW = 3 * TX;                     // tile box row (r, d, 1/diag, y): 96 values
static_assert(3 * (TX + 1 + XLEFT) <= PROW, "halo row");
static_assert(VX + XLEFT - 1 <= WROW, "voxel row");

enum { TOP_APPLY = 0, TOP_CHEB = 1, TOP_RESID = 2, TOP_DOT = 3 };

// tensor maps of one tiled launch: x (halo box), the voxel words, r, d, 1/diag and y (tile boxes)
struct TileMaps {
    CUtensorMap x, w, r, d, inv, y;
};

template <class T>
struct TileIO {
    float c1, c2;      // CHEB: d = c1 d + c2 D^-1 (r - K x)
    int raw;           // APPLY: keep held DOFs
    int partial;       // DOT: leave the step to the boundary-node kernel (st->pqPart holds the tiles' share)
};

__host__ __device__ constexpr uint32_t packTile(int tx, int ty, int tz) { return uint32_t(tx) | (uint32_t(ty) << 11) | (uint32_t(tz) << 22); }

// shared-memory layout of a tile CTA, every TMA destination on a 128-byte boundary: x halo, voxel
// words, the output tile (r for the smoother and residual epilogues, overwritten by y in place;
// a separate y tile otherwise), d (smoother, updated in place), 1/diag (smoother), the node masks
// and boundary list (32-bit) and two staging barriers (x and words; the epilogue operands)
__host__ __device__ constexpr size_t align128(size_t b) { return (b + 127) & ~size_t(127); }
__host__ __device__ constexpr bool tileHasR(int mode) { return mode == TOP_CHEB || mode == TOP_RESID; }
__host__ __device__ constexpr bool tileHasD(int mode) { return mode == TOP_CHEB; }
template <class T> __host__ __device__ constexpr size_t tileBytesX() { return sizeof(T) * PROW * HY * HZ; }
__host__ __device__ constexpr size_t tileBytesW() { return sizeof(uint32_t) * WROW * VY * VZ; }
template <class T> __host__ __device__ constexpr size_t tileBytesT() { return sizeof(T) * TROW * TY * TZ; }
template <class T> __host__ __device__ constexpr size_t tileOffW() { return align128(tileBytesX<T>()); }
template <class T> __host__ __device__ constexpr size_t tileOffY() { return tileOffW<T>() + align128(tileBytesW()); }
template <class T, int MODE> __host__ __device__ constexpr size_t tileOffD() {
    return tileOffY<T>() + align128(tileHasR(MODE) ? tileBytesT<float>() : tileBytesT<T>());
}
// INNER: the tile computes its boundary nodes itself (a compacted list in shared memory); else the
// boundary-node kernel does
template <class T, int MODE> __host__ __device__ constexpr size_t tileOffI() { return tileOffD<T, MODE>() + (tileHasD(MODE) ? align128(tileBytesT<float>()) : 0); }
template <class T, int MODE> __host__ __device__ constexpr size_t tileOffM() { return tileOffI<T, MODE>() + (tileHasD(MODE) ? align128(tileBytesT<float>()) : 0); }
template <class T, int MODE, bool INNER> __host__ __device__ constexpr size_t tileOffB() { return tileOffM<T, MODE>() + (INNER ? align128(TILE_NODES) : 0); }
template <class T, int MODE, bool INNER> __host__ __device__ constexpr size_t tileOffBar() {
    return tileOffB<T, MODE, INNER>() + (INNER ? align128(2 * TILE_NODES + 4 * 16) : 0);  // list, warp counts, chunk counter
}
template <class T, int MODE, bool INNER> __host__ __device__ constexpr size_t tileSmemBytes() { return tileOffBar<T, MODE, INNER>() + 16; }
// bytes each staging barrier expects
template <class T> __host__ __device__ constexpr unsigned tileStage0Bytes() { return unsigned(tileBytesX<T>() + tileBytesW()); }
template <int MODE> __host__ __device__ constexpr unsigned tileStage1Bytes() {
    return unsigned((tileHasR(MODE) ? tileBytesT<float>() : 0) + (tileHasD(MODE) ? 2 * tileBytesT<float>() : 0));
}

// ---- TMA and shared-memory barrier primitives (PTX, sm_90 and later; every copy lands in the issuing CTA's own shared memory)
__device__ __forceinline__ unsigned smemAddr(const void* p) { return unsigned(__cvta_generic_to_shared(p)); }
__device__ __forceinline__ void mbarInit(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smemAddr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbarExpectTx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smemAddr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbarTryWait(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smemAddr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait for the completion of the barrier phase with the given parity: false after `limit`
// polls (each poll may suspend the thread for a hardware-defined time)
__device__ __forceinline__ bool mbarWaitParity(uint64_t* bar, unsigned parity, unsigned limit) {
    for (unsigned it = 0; it < limit; it++)
        if (mbarTryWait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ bool mbarWait(uint64_t* bar, unsigned limit) { return mbarWaitParity(bar, 0, limit); }
// 3-D tiled load of a box at element coordinates (c0, c1, c2) into shared memory, completing on bar
__device__ __forceinline__ void tmaLoad3d(void* dst, const void* map, int c0, int c1, int c2, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(smemAddr(dst)),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(smemAddr(bar))
        : "memory");
}
// 3-D tiled store of a shared-memory box to (c0, c1, c2), c0..c2 >= 0; elements outside the tensor are skipped
__device__ __forceinline__ void tmaStore3d(const void* map, const void* src, int c0, int c1, int c2) {
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];\n" ::"l"(map), "r"(smemAddr(src)), "r"(c0),
                 "r"(c1), "r"(c2)
                 : "memory");
}
__device__ __forceinline__ void tmaStoreCommitWait() {
    asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
    asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
}
// makes this thread's shared-memory writes visible to later TMA (async proxy) reads
__device__ __forceinline__ void fenceAsyncShared() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// shared-memory offsets of x value (node tx + ox, ty + oy, tz + oz of the tile, component 0) and of
// the voxel word at tile voxel (vx, vy, vz) (voxel i0 - 1 + vx, ...)
__device__ __forceinline__ int xOff(int cx, int cy, int cz) { return ((cz + 1) * HY + (cy + 1)) * PROW + 3 * (cx + XLEFT); }
__device__ __forceinline__ int vOff(int vx, int vy, int vz) { return (vz * VY + vy) * WROW + vx + XLEFT - 1; }

template <class T, bool OWN16, bool DIFF>
struct TileOp {
    // adds voxel V's rows at a tile node to acc (V = di + 2 dj + 4 dk: the voxel at offset
    // (di - 1, dj - 1, dk - 1) from the node); A and B: rows oy = dj - 1 and dj (x offsets -1..1) of
    // the node's neighbourhood in planes oz = dk - 1 and dk (values already relative to the node's
    // own value when DIFF). V is a compile-time constant, so every Kb coefficient is a constant-bank
    // operand.
    template <int V>
    static __device__ __forceinline__ void voxel(const LevelView& L, const Coefs<T>& C, const uint32_t* vs, int cx, int cy, int cz,
                                                 const T (&A)[2][3][3], const T (&B)[2][3][3], T acc[3]) {
        constexpr int di = V & 1, dj = (V >> 1) & 1, dk = V >> 2;
        constexpr int a = cornerOf(1 - di, 1 - dj, 1 - dk);
        const uint32_t w = vs[vOff(cx + di, cy + dj, cz + dk)];
        if (w == 0) return;
        T xe[24];
#pragma unroll
        for (int b = 0; b < 8; b++) {
            const int bx = (b == 1 || b == 2 || b == 5 || b == 6), by = (b == 2 || b == 3 || b == 6 || b == 7), bz = b >> 2;
#pragma unroll
            for (int c = 0; c < 3; c++) xe[3 * b + c] = bz ? B[by][di + bx][c] : A[by][di + bx][c];
        }
        if (!(w & OWN_BIT)) {
            T t[3];
            kbRows<T>(C.Kb, a, xe, t);
            const T s = T(__uint_as_float(w));
            acc[0] += s * t[0];
            acc[1] += s * t[1];
            acc[2] += s * t[2];
        } else if (OWN16) {
            T t[3];
            own16Rows<T>(L.own16 + (long long)(w & ~OWN_BIT) * 576 + 72 * a, xe, t);
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
    // rows oy and oy + 1 (x offsets -1..1) of plane oz around tile node (cx, cy, cz), less own (DIFF)
    static __device__ __forceinline__ void rowPair(const T* xs, int cx, int cy, int cz, int oy, int oz, const T own[3], T (&R)[2][3][3]) {
#pragma unroll
        for (int yy = 0; yy < 2; yy++)
#pragma unroll
            for (int e = 0; e < 3; e++) {
                const T* xp = xs + xOff(cx + e - 1, cy + oy + yy, cz + oz);
                R[yy][e][0] = xp[0] - own[0];
                R[yy][e][1] = xp[1] - own[1];
                R[yy][e][2] = xp[2] - own[2];
            }
    }
    // K x at tile node (cx, cy, cz) by the per-voxel gather over its 8 voxels, two at a time: each
    // pair of voxels sharing (dj, dk) reads the two row pairs it needs (36 values live, not the 81
    // of the whole neighbourhood: fewer registers outweigh the extra shared-memory loads)
    static __device__ __forceinline__ void general(const LevelView& L, const Coefs<T>& C, const T* xs, const uint32_t* vs, int cx, int cy,
                                                   int cz, T acc[3], const T own[3]) {
        acc[0] = acc[1] = acc[2] = T(0);
        T A[2][3][3], B[2][3][3];
        rowPair(xs, cx, cy, cz, -1, -1, own, A);
        rowPair(xs, cx, cy, cz, -1, 0, own, B);
        voxel<0>(L, C, vs, cx, cy, cz, A, B, acc);
        voxel<1>(L, C, vs, cx, cy, cz, A, B, acc);
        rowPair(xs, cx, cy, cz, 0, -1, own, A);
        rowPair(xs, cx, cy, cz, 0, 0, own, B);
        voxel<2>(L, C, vs, cx, cy, cz, A, B, acc);
        voxel<3>(L, C, vs, cx, cy, cz, A, B, acc);
        rowPair(xs, cx, cy, cz, -1, 0, own, A);
        rowPair(xs, cx, cy, cz, -1, 1, own, B);
        voxel<4>(L, C, vs, cx, cy, cz, A, B, acc);
        voxel<5>(L, C, vs, cx, cy, cz, A, B, acc);
        rowPair(xs, cx, cy, cz, 0, 0, own, A);
        rowPair(xs, cx, cy, cz, 0, 1, own, B);
        voxel<6>(L, C, vs, cx, cy, cz, A, B, acc);
        voxel<7>(L, C, vs, cx, cy, cz, A, B, acc);
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

    // the same column sums with paired FMAs (__ffma2_rn, two nodes per instruction; each lane of
    // the pair rounds exactly like fmaf): nodes (0, 1) and (2, 3) of the column advance together,
    // fed by the pair of planes (p, p + 1) that the two nodes see at the same offset
    static __device__ __forceinline__ void column2(const Coefs32& C, const float* xs, int cx, int cy, float acc[TZ][3]) {
        static_assert(TZ == 4, "node pairs (0, 1) and (2, 3)");
        float2 A[2][3];
#pragma unroll
        for (int h = 0; h < 2; h++) A[h][0] = A[h][1] = A[h][2] = make_float2(0.f, 0.f);
#pragma unroll
        for (int p = -1; p <= 3; p++) {
            float2 v[9][3];
#pragma unroll
            for (int b = 0; b < 9; b++) {
                const float* x0 = xs + xOff(cx + b % 3 - 1, cy + b / 3 - 1, p);
                const float* x1 = xs + xOff(cx + b % 3 - 1, cy + b / 3 - 1, p + 1);
                v[b][0] = make_float2(x0[0], x1[0]);
                v[b][1] = make_float2(x0[1], x1[1]);
                v[b][2] = make_float2(x0[2], x1[2]);
            }
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int oz = p - 2 * h;  // pair h = nodes (2h, 2h + 1) sees planes (p, p + 1) at offset oz
                if (oz < -1 || oz > 1) continue;
#pragma unroll
                for (int b = 0; b < 9; b++) {
                    const int ox = b % 3 - 1, oy = b / 3 - 1, m = (ox + 1) + 3 * (oy + 1) + 9 * (oz + 1);
                    float2* a = A[h];
                    a[0] = __ffma2_rn(C.S2[m * 9 + 0], v[b][0], a[0]);
                    a[1] = __ffma2_rn(C.S2[m * 9 + 4], v[b][1], a[1]);
                    a[2] = __ffma2_rn(C.S2[m * 9 + 8], v[b][2], a[2]);
                    if (ox && oy) { a[0] = __ffma2_rn(C.S2[m * 9 + 1], v[b][1], a[0]); a[1] = __ffma2_rn(C.S2[m * 9 + 3], v[b][0], a[1]); }
                    if (ox && oz) { a[0] = __ffma2_rn(C.S2[m * 9 + 2], v[b][2], a[0]); a[2] = __ffma2_rn(C.S2[m * 9 + 6], v[b][0], a[2]); }
                    if (oy && oz) { a[1] = __ffma2_rn(C.S2[m * 9 + 5], v[b][2], a[1]); a[2] = __ffma2_rn(C.S2[m * 9 + 7], v[b][1], a[2]); }
                }
            }
        }
#pragma unroll
        for (int d = 0; d < 3; d++) {
            acc[0][d] = A[0][d].x;
            acc[1][d] = A[0][d].y;
            acc[2][d] = A[1][d].x;
            acc[3][d] = A[1][d].y;
        }
    }
};

}  // namespace dev
}  // namespace psfea
