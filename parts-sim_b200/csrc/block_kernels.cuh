// Device code of the multi-right-hand-side (block) solve. Included by solver.cu only.
//
// A block holds RB right-hand sides (RB = 8, 16 or 32) in the RHS-minor layout: value of DOF
// 3 n + d of right-hand side q at [(3 n + d) RB + q], over the level's pitched nodes n. One warp
// takes 32 / RB nodes, one lane per (node, right-hand side): the lanes of a node share its mask,
// coordinates, voxel words and element matrices (broadcast loads, read once for the whole block)
// and read their values as one contiguous RB-wide access per DOF. Kernels walk the level's list
// of active nodes, so empty regions cost nothing.
//
// Every right-hand side runs its own flexible CG (the reference's recurrence,
// native/src/fea/voxel_fea.cpp:863-927): the scalars rz, alpha, beta, the residual, the V-cycle's
// input scale and the stop decision are per right-hand side (BlockState). A finished right-hand
// side keeps its iterate: its step length is 0 and its V-cycle input is 0. Reductions are
// deterministic (lane-wise partial sums per block, folded in block order by the last block).
#pragma once

#include "kernels.cuh"

namespace psfea {
namespace dev {

constexpr int RBMAX = 32;
constexpr int BLOCK_THREADS = 256;

// per right-hand side control of a block solve
struct BlockState {
    double bnorm[RBMAX], rel[RBMAX], rz[RBMAX], alpha[RBMAX], beta[RBMAX], rmax[RBMAX], scale[RBMAX], vscale[RBMAX], pq[RBMAX];
    int it[RBMAX], done[RBMAX], status[RBMAX];
    double tol;
    int iter, maxIter, first, allDone, nrhs;
};

// Lane-wise grid reduction: lane l holds K values of right-hand side l % RB. Returns true in the
// last block to finish, where thread t < RB holds in out[] the totals of right-hand side t (sums,
// or maxima for the bits of maxMask). partials: gridDim.x * RB * K doubles; ticket starts at 0 and
// is left at 0. Sums run in a fixed order (warp lanes, warps, blocks), so results are reproducible.
template <int K, int RB>
__device__ bool laneGridReduce(double (&v)[K], unsigned maxMask, double* partials, unsigned* ticket, double (&out)[K]) {
    constexpr int NW = BLOCK_THREADS / 32;
    __shared__ double sh[NW * RBMAX * K];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = RB; o < 32; o <<= 1)
#pragma unroll
        for (int c = 0; c < K; c++) {
            const double w = __shfl_xor_sync(0xffffffffu, v[c], o);
            v[c] = ((maxMask >> c) & 1) ? fmax(v[c], w) : v[c] + w;
        }
    if (lane < RB)
#pragma unroll
        for (int c = 0; c < K; c++) sh[(wid * RB + lane) * K + c] = v[c];
    __syncthreads();
    if (threadIdx.x < RB) {
        double a[K];
#pragma unroll
        for (int c = 0; c < K; c++) a[c] = 0;
        for (int w = 0; w < NW; w++)
#pragma unroll
            for (int c = 0; c < K; c++) {
                const double p = sh[(w * RB + threadIdx.x) * K + c];
                a[c] = ((maxMask >> c) & 1) ? fmax(a[c], p) : a[c] + p;
            }
#pragma unroll
        for (int c = 0; c < K; c++) partials[((size_t)blockIdx.x * RB + threadIdx.x) * K + c] = a[c];
        __threadfence();
    }
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return false;
    __threadfence();
    // the last block: thread t sums right-hand side t % RB over the blocks b = t / RB (mod NC)
    constexpr int NC = BLOCK_THREADS / RB;
    const int q = threadIdx.x % RB, chunk = threadIdx.x / RB;
    double a[K];
#pragma unroll
    for (int c = 0; c < K; c++) a[c] = 0;
    for (unsigned b = chunk; b < gridDim.x; b += NC)
#pragma unroll
        for (int c = 0; c < K; c++) {
            const double p = __ldcg(partials + ((size_t)b * RB + q) * K + c);
            a[c] = ((maxMask >> c) & 1) ? fmax(a[c], p) : a[c] + p;
        }
    __syncthreads();  // sh is reused
#pragma unroll
    for (int c = 0; c < K; c++) sh[(chunk * RB + q) * K + c] = a[c];
    __syncthreads();
    if (threadIdx.x < RB) {
#pragma unroll
        for (int c = 0; c < K; c++) out[c] = 0;
        for (int ch = 0; ch < NC; ch++)
#pragma unroll
            for (int c = 0; c < K; c++) {
                const double p = sh[(ch * RB + threadIdx.x) * K + c];
                out[c] = ((maxMask >> c) & 1) ? fmax(out[c], p) : out[c] + p;
            }
    }
    if (threadIdx.x == 0) *ticket = 0;
    return true;
}

// the running state of a right-hand side
__device__ __forceinline__ bool rhsRunning(const BlockState* bs, int q) { return q < bs->nrhs && !bs->done[q]; }

// after a per-right-hand-side stop decision: the whole block is done when every one is (thread 0
// of the last block, after the threads t < RB have written their decisions)
__device__ __forceinline__ void blockAllDone(BlockState* bs) {
    int all = 1;
    for (int q = 0; q < bs->nrhs; q++) all &= bs->done[q] != 0;
    bs->allDone = all;
}

enum { BOP_APPLY = 0, BOP_CHEB = 1, BOP_RESID = 2, BOP_DOT = 3 };

// (K x) at node (i, j, k) of a block vector (stride S, x at the lane's right-hand side) with each of
// the node's 27 neighbours read once, two z-planes of 9 nodes in registers at a time (planes -1 and
// 0 for the voxels below the node, 0 and +1 for those above): the same sums in the same order as
// applyAt (so bitwise the same), with 81 loads instead of up to 192 on nodes that take the per-voxel
// gather. Neighbours outside the grid read 0; they only ever meet empty voxels.
// V: the storage type of x (T, or __half for the FP16 coarse-level vectors; converted on load).
template <class T, bool OWN16, int S, bool SMEM = false, class V = T>
__device__ __forceinline__ void applyNbr(const LevelView& L, const Coefs<T>& C, const V* __restrict__ x, int i, int j, int k, long long n,
                                         uint8_t mask, T acc[3]) {
    acc[0] = acc[1] = acc[2] = T(0);
    if (!(mask & NM_ACTIVE)) return;
    const long long NX = L.PX, NXY = (long long)L.PX * L.NY;
    auto plane = [&](int oz, T (&P)[9][3]) {
#pragma unroll
        for (int b = 0; b < 9; b++) {
            const int ox = b % 3 - 1, oy = b / 3 - 1;
            const bool in = i + ox >= 0 && j + oy >= 0 && k + oz >= 0 && i + ox < L.NX && j + oy < L.NY && k + oz < L.NZ;
            const V* xp = x + 3 * S * (n + ox + oy * NX + oz * NXY);
            P[b][0] = in ? ldv<T>(xp) : T(0);
            P[b][1] = in ? ldv<T>(xp + S) : T(0);
            P[b][2] = in ? ldv<T>(xp + 2 * S) : T(0);
        }
    };
    T A[9][3], B[9][3];  // A: planes -1 then +1; B: plane 0
    plane(-1, A);
    plane(0, B);
    const T own[3] = {B[4][0], B[4][1], B[4][2]};
    if (mask & NM_UNIFORM) {
        const float s = __uint_as_float(__ldg(L.word + L.wi(i - 1, j - 1, k - 1)));
        T a0 = 0, a1 = 0, a2 = 0;
        auto sweep = [&](int oz, const T (&P)[9][3]) {
#pragma unroll
            for (int b = 0; b < 9; b++) {
                const int ox = b % 3 - 1, oy = b / 3 - 1, m = b + 9 * (oz + 1);
                const T x0 = P[b][0], x1 = P[b][1], x2 = P[b][2];
                a0 += C.S[m * 9 + 0] * x0;
                a1 += C.S[m * 9 + 4] * x1;
                a2 += C.S[m * 9 + 8] * x2;
                if (ox && oy) { a0 += C.S[m * 9 + 1] * x1; a1 += C.S[m * 9 + 3] * x0; }
                if (ox && oz) { a0 += C.S[m * 9 + 2] * x2; a2 += C.S[m * 9 + 6] * x0; }
                if (oy && oz) { a1 += C.S[m * 9 + 5] * x2; a2 += C.S[m * 9 + 7] * x1; }
            }
        };
        sweep(-1, A);
        sweep(0, B);
        plane(1, A);
        sweep(1, A);
        acc[0] = T(s) * a0;
        acc[1] = T(s) * a1;
        acc[2] = T(s) * a2;
    } else {
        // voxel vv = di + 2 dj + 4 dk at offset (di - 1, dj - 1, dk - 1); its corner b sits in plane
        // dk + bz - 1: lo = the plane below (dk - 1), hi = the plane above (dk)
        auto voxel = [&](int vv, const T (&lo)[9][3], const T (&hi)[9][3]) {
            const int di = vv & 1, dj = (vv >> 1) & 1, dk = vv >> 2;
            const int ei = i - 1 + di, ej = j - 1 + dj, ek = k - 1 + dk;
            if (ei < 0 || ej < 0 || ek < 0 || ei >= L.nx || ej >= L.ny || ek >= L.nz) return;
            const uint32_t w = __ldg(L.word + L.wi(ei, ej, ek));
            if (w == 0) return;
            const int a = cornerOf(1 - di, 1 - dj, 1 - dk);
            T xe[24];
#pragma unroll
            for (int b = 0; b < 8; b++) {
                const int bx = (b == 1 || b == 2 || b == 5 || b == 6), by = (b == 2 || b == 3 || b == 6 || b == 7), bz = b >> 2;
                const int b9 = (di + bx) + 3 * (dj + by);
                const T* src = bz ? hi[b9] : lo[b9];
                xe[3 * b] = src[0];
                xe[3 * b + 1] = src[1];
                xe[3 * b + 2] = src[2];
            }
            if (!(w & OWN_BIT)) {
                T t[3];
                kbRows<T>(C.Kb, a, xe, t);
                const T sc = T(__uint_as_float(w));
                acc[0] += sc * t[0];
                acc[1] += sc * t[1];
                acc[2] += sc * t[2];
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
        };
#pragma unroll
        for (int vv = 0; vv < 4; vv++) voxel(vv, A, B);
        plane(1, A);
#pragma unroll
        for (int vv = 4; vv < 8; vv++) voxel(vv, B, A);
    }
    if (L.dadd) {
#pragma unroll
        for (int d = 0; d < 3; d++) acc[d] += (sizeof(T) == 8 ? T(L.dadd[3 * n + d]) : T(L.dadd32[3 * n + d])) * own[d];
    }
}

// One pass over the level's active nodes of y = K x for every right-hand side, with a per-DOF epilogue:
//   BOP_APPLY  y = K x (held DOFs 0 unless raw)
//   BOP_CHEB   d = c1 d + c2 D^-1 (r - K x); y = x + d        (Chebyshev / Jacobi step, 32-bit)
//   BOP_RESID  y = r - K x
//   BOP_DOT    y = K x (held 0) and each right-hand side's CG step alpha = rz / (x . y); x . y <= 0
//              ends that right-hand side as a breakdown (voxel_fea.cpp:902-905)
// The product is the single-vector one (applyAt, voxel_fea.cpp:422-486) with the block's stride.
// The block path's assembled stencils are node-major: node t's row at t * STN_ROW holds its 27 3x3
// blocks with the neighbours taken in pairs (m, m + 1) = (2 P, 2 P + 1), P = 0..13 (m = (ox + 1) +
// 3 (oy + 1) + 9 (oz + 1); the 28th slot is 0): entry (p, q) of the pair's two blocks side by side
// at 18 P + 2 (3 p + q) + (m & 1). A warp copies its nodes' rows into shared memory with 16-byte
// loads (512 contiguous bytes per instruction) and every lane of a node reads them as broadcasts;
// one paired FMA then advances both neighbours of a pair: 126 paired FMAs per node and right-hand
// side where the per-voxel gather takes 288 (576 multiply-adds), the coefficients read from HBM
// once per node for the whole block.
constexpr int STN_ROW = 252;
__host__ __device__ constexpr int stnPairAt(int m, int p, int q) { return 18 * (m >> 1) + 2 * (3 * p + q) + (m & 1); }
template <class T>
__host__ __device__ constexpr size_t stnBlockSmem(int npw) { return size_t(BLOCK_THREADS / 32) * npw * STN_ROW * sizeof(T); }

template <class T, int S>
__device__ __forceinline__ void stnBlock(const LevelView& L, const T* __restrict__ row, const T* __restrict__ x, long long n, int i, int j,
                                         int k, T acc[3]) {
    static_assert(sizeof(T) == 4, "the paired layout is FP32");
    const long long NX = L.PX, NXY = (long long)L.PX * L.NY;
    auto xOf = [&](int m, float (&v)[3]) {
        const int ox = m % 3 - 1, oy = (m / 3) % 3 - 1, oz = m / 9 - 1;
        const bool in = m < 27 && i + ox >= 0 && j + oy >= 0 && k + oz >= 0 && i + ox < L.NX && j + oy < L.NY && k + oz < L.NZ;
        const T* xp = x + 3 * S * (n + ox + oy * NX + oz * NXY);
        v[0] = in ? __ldg(xp) : 0.f;
        v[1] = in ? __ldg(xp + S) : 0.f;
        v[2] = in ? __ldg(xp + 2 * S) : 0.f;
    };
    const float4* R = reinterpret_cast<const float4*>(row);
    float2 a2[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
    float4 cf = make_float4(0.f, 0.f, 0.f, 0.f);
    int have = -1;
#pragma unroll
    for (int P = 0; P < 14; P++) {
        float u[3], w[3];
        xOf(2 * P, u);
        xOf(2 * P + 1, w);
#pragma unroll
        for (int e = 0; e < 9; e++) {
            const int f = 18 * P + 2 * e;  // the pair's entry (p, q) = (e / 3, e % 3): floats f, f + 1
            if (f / 4 != have) {
                have = f / 4;
                cf = R[have];
            }
            const float2 b = (f % 4 == 0) ? make_float2(cf.x, cf.y) : make_float2(cf.z, cf.w);
            a2[e / 3] = __ffma2_rn(b, make_float2(u[e % 3], w[e % 3]), a2[e / 3]);
        }
    }
    acc[0] = a2[0].x + a2[0].y;
    acc[1] = a2[1].x + a2[1].y;
    acc[2] = a2[2].x + a2[2].y;
}

// STN: the product from the level's assembled stencils (stn, over act) instead of the gather.
template <class T, int MODE, bool OWN16, int RB, bool STN = false>
__global__ void __launch_bounds__(BLOCK_THREADS, 2) kb_op(LevelView L, Coefs<T> C, const int* __restrict__ act, int nAct,
                                                       const T* __restrict__ stn, const T* __restrict__ x, T* __restrict__ y,
                                                       const float* __restrict__ r, float* __restrict__ d, float c1, float c2, int raw,
                                                       BlockState* bs, double* partials, unsigned* ticket, Ctl ctl) {
    if (skipped(ctl)) return;
    constexpr int NPW = 32 / RB;
    const int lane = threadIdx.x & 31, q = lane % RB, sub = lane / RB;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((long long)gridDim.x * blockDim.x) >> 5;
    extern __shared__ __align__(16) unsigned char kbRaw[];
    T* rows = reinterpret_cast<T*>(kbRaw) + (threadIdx.x >> 5) * NPW * STN_ROW;  // this warp's NPW stencil rows
    double dot[1] = {0.0};
    // warp-uniform sweep (the stencil rows are shared within the warp); lanes past the list idle
    for (long long tb = warp * NPW; tb < nAct; tb += nw * NPW) {
        const long long t = tb + sub;
        if constexpr (STN) {
            constexpr int VP = 16 / int(sizeof(T)), PIECES = STN_ROW / VP;  // 16-byte pieces of a row
            for (int e = lane; e < NPW * PIECES; e += 32) {
                const int u = e / PIECES, g = e - u * PIECES;
                if (tb + u < nAct) {
                    const uint4 v = __ldcs(reinterpret_cast<const uint4*>(stn + (tb + u) * STN_ROW) + g);
                    reinterpret_cast<uint4*>(rows + u * STN_ROW)[g] = v;
                }
            }
            __syncwarp();
        }
        if (t < nAct) {
            const long long n = act[t];
            const uint8_t mask = __ldg(L.nmask + n);
            int i, j, k;
            nodeCoords(L, n, i, j, k);
            T acc[3];
            if constexpr (STN) stnBlock<T, RB>(L, rows + sub * STN_ROW, x + q, n, i, j, k, acc);
            else applyNbr<T, OWN16, RB>(L, C, x + q, i, j, k, n, mask, acc);
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const long long id = (3 * n + c) * RB + q;
                const bool fx = fixedDof(mask, c);
                if constexpr (MODE == BOP_APPLY) {
                    y[id] = (!raw && fx) ? T(0) : acc[c];
                } else if constexpr (MODE == BOP_DOT) {
                    const T yv = fx ? T(0) : acc[c];
                    y[id] = yv;
                    dot[0] += double(x[id]) * double(yv);
                } else if constexpr (MODE == BOP_RESID) {
                    y[id] = fx ? T(0) : T(r[id]) - acc[c];
                } else {
                    if (fx) {
                        d[id] = 0.f;
                        y[id] = T(0);
                    } else {
                        const float dn = c1 * d[id] + c2 * __ldg(L.invD + 3 * n + c) * (r[id] - float(acc[c]));
                        d[id] = dn;
                        y[id] = x[id] + T(dn);
                    }
                }
            }
        }
        if constexpr (STN) __syncwarp();  // the rows are refilled next
    }
    if constexpr (MODE == BOP_DOT) {
        double tot[1];
        if (laneGridReduce<1, RB>(dot, 0u, partials, ticket, tot)) {
            const int qq = threadIdx.x;
            if (qq < RB) {
                bs->pq[qq] = tot[0];
                if (!rhsRunning(bs, qq)) {
                    bs->alpha[qq] = 0;
                } else if (!(tot[0] > 0)) {
                    bs->alpha[qq] = 0;
                    bs->status[qq] = ST_BREAKDOWN;
                    bs->done[qq] = 1;
                    bs->it[qq] = bs->iter;
                } else {
                    bs->alpha[qq] = bs->rz[qq] / tot[0];
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) blockAllDone(bs);
        }
    }
}

// z = d = c0 D^-1 r (the first Chebyshev step from zero) at the active nodes
template <int RB>
__global__ void kb_cheb_first(const int* __restrict__ act, int nAct, const float* __restrict__ invD, const float* __restrict__ r,
                              float* __restrict__ d, float* __restrict__ z, float c0, Ctl ctl) {
    if (skipped(ctl)) return;
    const long long total = (long long)nAct * 3 * RB;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const long long t = e / (3 * RB);
        const int rem = int(e - t * 3 * RB), c = rem / RB, q = rem - c * RB;
        const long long dof = 3 * (long long)act[t] + c, id = dof * RB + q;
        const float v = c0 * __ldg(invD + dof) * r[id];
        d[id] = v;
        z[id] = v;
    }
}

// rc = P^T rf at the coarse level's active nodes (fine 2I weight 1, 2I +- 1 weight 1/2 per axis),
// held coarse DOFs 0; with dc, the coarse level's first smoothing step d = z = c0 D^-1 rc
template <int RB>
__global__ void kb_restrict(LevelView F, LevelView C, const int* __restrict__ cAct, int nCAct, const float* __restrict__ rf,
                            float* __restrict__ rc, float* __restrict__ dc, float* __restrict__ zc, float c0, Ctl ctl) {
    if (skipped(ctl)) return;
    constexpr int NPW = 32 / RB;
    const int lane = threadIdx.x & 31, q = lane % RB, sub = lane / RB;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long FPX = F.PX, FPXY = (long long)F.PX * F.NY;
    for (long long t = warp * NPW + sub; t < nCAct; t += nw * NPW) {
        const long long cn = cAct[t];
        const uint8_t mask = C.nmask[cn];
        int I, J, K;
        nodeCoords(C, cn, I, J, K);
        float s0 = 0, s1 = 0, s2 = 0;
        for (int dk = -1; dk <= 1; dk++) {
            const int k = 2 * K + dk;
            if (k < 0 || k >= F.NZ) continue;
            const float wk = dk ? 0.5f : 1.f;
            for (int dj = -1; dj <= 1; dj++) {
                const int j = 2 * J + dj;
                if (j < 0 || j >= F.NY) continue;
                const float wj = (dj ? 0.5f : 1.f) * wk;
                for (int di = -1; di <= 1; di++) {
                    const int i = 2 * I + di;
                    if (i < 0 || i >= F.NX) continue;
                    const float w = (di ? 0.5f : 1.f) * wj;
                    const float* p = rf + 3 * RB * (i + j * FPX + k * FPXY) + q;
                    s0 += w * p[0];
                    s1 += w * p[RB];
                    s2 += w * p[2 * RB];
                }
            }
        }
        const float sv[3] = {s0, s1, s2};
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const long long id = (3 * cn + c) * RB + q;
            const float v = fixedDof(mask, c) ? 0.f : sv[c];
            rc[id] = v;
            if (dc) {
                const float dv = c0 * __ldg(C.invD + 3 * cn + c) * v;
                dc[id] = dv;
                zc[id] = dv;
            }
        }
    }
}

// zf += P zc at the free DOFs of the fine level's active nodes (trilinear)
template <int RB>
__global__ void kb_prolong(LevelView F, int CPX, int CNY, const int* __restrict__ fAct, int nFAct, const float* __restrict__ zc,
                           float* __restrict__ zf, Ctl ctl) {
    if (skipped(ctl)) return;
    constexpr int NPW = 32 / RB;
    const int lane = threadIdx.x & 31, q = lane % RB, sub = lane / RB;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long CNX = CPX, CNXY = (long long)CPX * CNY;
    for (long long t = warp * NPW + sub; t < nFAct; t += nw * NPW) {
        const long long fn = fAct[t];
        const uint8_t mask = F.nmask[fn];
        if ((mask & 7) == 7) continue;
        int i, j, k;
        nodeCoords(F, fn, i, j, k);
        const int i0 = i >> 1, j0 = j >> 1, k0 = k >> 1;
        const int ni = (i & 1) ? 2 : 1, nj = (j & 1) ? 2 : 1, nk = (k & 1) ? 2 : 1;
        const float w = ((i & 1) ? 0.5f : 1.f) * ((j & 1) ? 0.5f : 1.f) * ((k & 1) ? 0.5f : 1.f);
        float s0 = 0, s1 = 0, s2 = 0;
        for (int c = 0; c < nk; c++)
            for (int b = 0; b < nj; b++)
                for (int a = 0; a < ni; a++) {
                    const float* p = zc + 3 * RB * ((i0 + a) + (j0 + b) * CNX + (k0 + c) * CNXY) + q;
                    s0 += w * p[0];
                    s1 += w * p[RB];
                    s2 += w * p[2 * RB];
                }
        float* o = zf + 3 * RB * fn + q;
        if (!fixedDof(mask, 0)) o[0] += s0;
        if (!fixedDof(mask, 1)) o[RB] += s1;
        if (!fixedDof(mask, 2)) o[2 * RB] += s2;
    }
}

// coarsest level: z = A^-1 r over the m free DOFs for every right-hand side (FP64 dense inverse,
// one row per lane group; the row's entries are read once for the group's right-hand sides)
template <class TI, class TO, int RB>
__global__ void kb_coarse(int m, const int* __restrict__ dof, const double* __restrict__ Ainv, const TI* __restrict__ r, TO* __restrict__ z,
                          Ctl ctl) {
    if (skipped(ctl)) return;
    constexpr int NPW = 32 / RB;
    const int lane = threadIdx.x & 31, q = lane % RB, sub = lane / RB;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long row = warp * NPW + sub; row < m; row += nw * NPW) {
        const double* a = Ainv + (size_t)row * m;
        double s0 = 0, s1 = 0;
        int c = 0;
        for (; c + 1 < m; c += 2) {
            s0 += a[c] * double(r[(long long)dof[c] * RB + q]);
            s1 += a[c + 1] * double(r[(long long)dof[c + 1] * RB + q]);
        }
        if (c < m) s0 += a[c] * double(r[(long long)dof[c] * RB + q]);
        z[(long long)dof[row] * RB + q] = TO(s0 + s1);
    }
}

// ---------------------------------------------------------------- block CG vector kernels (FP64)

// r = f - K x at free DOFs; bnorm = ||f_free||, rel = ||r|| / bnorm, rmax = max |r_free| per
// right-hand side (voxel_fea.cpp:876-886); a zero load ends its right-hand side with u = 0
template <int RB>
__global__ void kb_cg_init(const int* __restrict__ act, int nAct, const uint8_t* __restrict__ nmask, const double* __restrict__ f,
                           const double* __restrict__ kx, double* __restrict__ r, BlockState* bs, double* partials, unsigned* ticket) {
    constexpr int NPW = 32 / RB;
    const int lane = threadIdx.x & 31, q = lane % RB, sub = lane / RB;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((long long)gridDim.x * blockDim.x) >> 5;
    double v[3] = {0, 0, 0};
    for (long long t = warp * NPW + sub; t < nAct; t += nw * NPW) {
        const long long n = act[t];
        const uint8_t mask = nmask[n];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const long long id = (3 * n + c) * RB + q;
            double rv = 0;
            if (!fixedDof(mask, c)) {
                const double fv = f[id];
                rv = fv - kx[id];
                v[0] += fv * fv;
                v[1] += rv * rv;
                v[2] = fmax(v[2], fabs(rv));
            }
            r[id] = rv;
        }
    }
    double tot[3];
    if (laneGridReduce<3, RB>(v, 4u, partials, ticket, tot)) {
        const int qq = threadIdx.x;
        if (qq < RB) {
            bs->bnorm[qq] = sqrt(tot[0]);
            bs->rmax[qq] = tot[2];
            bs->scale[qq] = tot[2] > 0 ? 1.0 / tot[2] : 1.0;
            bs->it[qq] = 0;
            bs->status[qq] = ST_RUNNING;
            bs->alpha[qq] = 0;
            if (qq >= bs->nrhs) {
                bs->rel[qq] = 0;
                bs->done[qq] = 1;
            } else if (bs->bnorm[qq] == 0) {
                bs->rel[qq] = 0;
                bs->status[qq] = ST_CONVERGED;
                bs->done[qq] = 2;  // zero load: the solution is zero
            } else {
                bs->rel[qq] = sqrt(tot[1]) / bs->bnorm[qq];
                bs->done[qq] = 0;
                if (bs->rel[qq] <= bs->tol) {
                    bs->status[qq] = ST_CONVERGED;
                    bs->done[qq] = 1;
                } else if (bs->maxIter <= 0) {
                    bs->status[qq] = ST_MAXITER;
                    bs->done[qq] = 1;
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) blockAllDone(bs);
    }
}

// x += alpha p, r -= alpha q at free DOFs of running right-hand sides; rel, rmax per right-hand
// side; stop on rel <= tol or the cap. Fused: the V-cycle input r32 = r * scale (0 for finished
// right-hand sides) and the finest level's first Chebyshev step d = z = c0 D^-1 r32.
template <int RB>
__global__ void kb_cg_update(const int* __restrict__ act, int nAct, const uint8_t* __restrict__ nmask, double* __restrict__ x,
                             double* __restrict__ r, const double* __restrict__ p, const double* __restrict__ kp, float* __restrict__ r32,
                             const float* __restrict__ invD, float* __restrict__ d, float* __restrict__ z, float c0, BlockState* bs,
                             double* partials, unsigned* ticket, Ctl ctl) {
    if (skipped(ctl)) return;
    constexpr int NPW = 32 / RB;
    const int lane = threadIdx.x & 31, q = lane % RB, sub = lane / RB;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((long long)gridDim.x * blockDim.x) >> 5;
    const bool run = rhsRunning(bs, q);
    const double alpha = bs->alpha[q], s = bs->scale[q];
    double v[2] = {0, 0};
    for (long long t = warp * NPW + sub; t < nAct; t += nw * NPW) {
        const long long n = act[t];
        const uint8_t mask = nmask[n];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            if (fixedDof(mask, c)) continue;
            const long long id = (3 * n + c) * RB + q;
            float rs = 0.f;
            if (run) {
                x[id] += alpha * p[id];
                const double rv = r[id] - alpha * kp[id];
                r[id] = rv;
                v[0] += rv * rv;
                v[1] = fmax(v[1], fabs(rv));
                rs = float(rv * s);
            }
            r32[id] = rs;
            const float dv = c0 * __ldg(invD + 3 * n + c) * rs;
            d[id] = dv;
            z[id] = dv;
        }
    }
    double tot[2];
    if (laneGridReduce<2, RB>(v, 2u, partials, ticket, tot)) {
        const int qq = threadIdx.x;
        if (qq < RB && rhsRunning(bs, qq)) {
            bs->rel[qq] = sqrt(tot[0]) / bs->bnorm[qq];
            bs->vscale[qq] = bs->scale[qq];
            bs->rmax[qq] = tot[1];
            bs->scale[qq] = tot[1] > 0 ? 1.0 / tot[1] : 1.0;
            bs->it[qq] = bs->iter + 1;
            if (bs->rel[qq] <= bs->tol) {
                bs->status[qq] = ST_CONVERGED;
                bs->done[qq] = 1;
            } else if (bs->iter + 1 >= bs->maxIter) {
                bs->status[qq] = ST_MAXITER;
                bs->done[qq] = 1;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            bs->iter += 1;
            blockAllDone(bs);
        }
    }
}

// the V-cycle input of every running right-hand side, r32 = float(r / max|r_free|) (voxel_fea.cpp:
// 856-857), and the first Chebyshev step d = z = c0 D^-1 r32; 0 for finished ones
template <int RB>
__global__ void kb_vc_load(const int* __restrict__ act, int nAct, const uint8_t* __restrict__ nmask, const double* __restrict__ r,
                           float* __restrict__ r32, const float* __restrict__ invD, float* __restrict__ d, float* __restrict__ z, float c0,
                           BlockState* bs, Ctl ctl) {
    if (skipped(ctl)) return;
    constexpr int NPW = 32 / RB;
    const int lane = threadIdx.x & 31, q = lane % RB, sub = lane / RB;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((long long)gridDim.x * blockDim.x) >> 5;
    const bool run = rhsRunning(bs, q);
    const double s = bs->scale[q];
    for (long long t = warp * NPW + sub; t < nAct; t += nw * NPW) {
        const long long n = act[t];
        const uint8_t mask = nmask[n];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            if (fixedDof(mask, c)) continue;
            const long long id = (3 * n + c) * RB + q;
            const float rs = run ? float(r[id] * s) : 0.f;
            r32[id] = rs;
            const float dv = c0 * __ldg(invD + 3 * n + c) * rs;
            d[id] = dv;
            z[id] = dv;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x < RB) bs->vscale[threadIdx.x] = bs->scale[threadIdx.x];
}

// z = z32 / vscale; rzNew = r.z, zq = z.(K p) per running right-hand side; beta = max(0, -alpha
// zq / rz) (voxel_fea.cpp:913-917), 0 on the first pass
template <int RB>
__global__ void kb_cg_dots(const int* __restrict__ act, int nAct, const uint8_t* __restrict__ nmask, const double* __restrict__ r,
                           const float* __restrict__ z32, const double* __restrict__ z64, const double* __restrict__ kp, BlockState* bs,
                           double* partials, unsigned* ticket, Ctl ctl) {
    if (skipped(ctl)) return;
    constexpr int NPW = 32 / RB;
    const int lane = threadIdx.x & 31, q = lane % RB, sub = lane / RB;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((long long)gridDim.x * blockDim.x) >> 5;
    const bool run = rhsRunning(bs, q), first = bs->first;
    const double inv = 1.0 / bs->vscale[q];
    double v[2] = {0, 0};
    if (run)
        for (long long t = warp * NPW + sub; t < nAct; t += nw * NPW) {
            const long long n = act[t];
            const uint8_t mask = nmask[n];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                if (fixedDof(mask, c)) continue;
                const long long id = (3 * n + c) * RB + q;
                const double zv = z64 ? z64[id] : double(z32[id]) * inv;
                v[0] += r[id] * zv;
                if (!first) v[1] += zv * kp[id];
            }
        }
    double tot[2];
    if (laneGridReduce<2, RB>(v, 0u, partials, ticket, tot)) {
        const int qq = threadIdx.x;
        if (qq < RB && rhsRunning(bs, qq)) {
            bs->beta[qq] = first ? 0.0 : fmax(0.0, -bs->alpha[qq] * tot[1] / bs->rz[qq]);
            bs->rz[qq] = tot[0];
        }
    }
}

// p = z + beta p at free DOFs of running right-hand sides
template <int RB>
__global__ void kb_cg_p(const int* __restrict__ act, int nAct, const uint8_t* __restrict__ nmask, const float* __restrict__ z32,
                        const double* __restrict__ z64, double* __restrict__ p, const BlockState* bs, Ctl ctl) {
    if (skipped(ctl)) return;
    constexpr int NPW = 32 / RB;
    const int lane = threadIdx.x & 31, q = lane % RB, sub = lane / RB;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((long long)gridDim.x * blockDim.x) >> 5;
    if (!rhsRunning(bs, q)) return;
    const double inv = 1.0 / bs->vscale[q], beta = bs->beta[q];
    const bool first = bs->first;
    for (long long t = warp * NPW + sub; t < nAct; t += nw * NPW) {
        const long long n = act[t];
        const uint8_t mask = nmask[n];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            if (fixedDof(mask, c)) continue;
            const long long id = (3 * n + c) * RB + q;
            const double zv = z64 ? z64[id] : double(z32[id]) * inv;
            p[id] = first ? zv : zv + beta * p[id];
        }
    }
}

__global__ void kb_clear_first(BlockState* bs) { bs->first = 0; }

// true residual per right-hand side after the loop: ||f - K x||_free / bnorm (voxel_fea.cpp:921-925)
template <int RB>
__global__ void kb_final(const int* __restrict__ act, int nAct, const uint8_t* __restrict__ nmask, const double* __restrict__ f,
                         const double* __restrict__ kx, BlockState* bs, double* partials, unsigned* ticket) {
    constexpr int NPW = 32 / RB;
    const int lane = threadIdx.x & 31, q = lane % RB, sub = lane / RB;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((long long)gridDim.x * blockDim.x) >> 5;
    double v[1] = {0};
    for (long long t = warp * NPW + sub; t < nAct; t += nw * NPW) {
        const long long n = act[t];
        const uint8_t mask = nmask[n];
#pragma unroll
        for (int c = 0; c < 3; c++)
            if (!fixedDof(mask, c)) {
                const long long id = (3 * n + c) * RB + q;
                const double rv = f[id] - kx[id];
                v[0] += rv * rv;
            }
    }
    double tot[1];
    if (laneGridReduce<1, RB>(v, 0u, partials, ticket, tot)) {
        const int qq = threadIdx.x;
        if (qq < RB && qq < bs->nrhs) bs->rel[qq] = bs->bnorm[qq] > 0 ? sqrt(tot[0]) / bs->bnorm[qq] : 0.0;
    }
}

// max |r_free| per right-hand side into rmax / scale (the block preconditioner's entry)
template <int RB>
__global__ void kb_rmax(const int* __restrict__ act, int nAct, const uint8_t* __restrict__ nmask, const double* __restrict__ r, BlockState* bs,
                        double* partials, unsigned* ticket) {
    constexpr int NPW = 32 / RB;
    const int lane = threadIdx.x & 31, q = lane % RB, sub = lane / RB;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((long long)gridDim.x * blockDim.x) >> 5;
    double v[1] = {0};
    for (long long t = warp * NPW + sub; t < nAct; t += nw * NPW) {
        const long long n = act[t];
        const uint8_t mask = nmask[n];
#pragma unroll
        for (int c = 0; c < 3; c++)
            if (!fixedDof(mask, c)) v[0] = fmax(v[0], fabs(r[(3 * n + c) * RB + q]));
    }
    double tot[1];
    if (laneGridReduce<1, RB>(v, 1u, partials, ticket, tot)) {
        const int qq = threadIdx.x;
        if (qq < RB) {
            bs->rmax[qq] = tot[0];
            bs->scale[qq] = tot[0] > 0 ? 1.0 / tot[0] : 1.0;
            bs->done[qq] = (qq < bs->nrhs && tot[0] > 0) ? 0 : 1;  // a zero vector gives z = 0
        }
    }
}

// z = z32 / vscale at active nodes (voxel_fea.cpp:859-860), 0 for finished right-hand sides
template <int RB>
__global__ void kb_vc_store(const int* __restrict__ act, int nAct, const float* __restrict__ z32, double* __restrict__ z, const BlockState* bs) {
    const long long total = (long long)nAct * 3 * RB;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const long long t = e / (3 * RB);
        const int rem = int(e - t * 3 * RB), c = rem / RB, q = rem - c * RB;
        const long long id = (3 * (long long)act[t] + c) * RB + q;
        z[id] = rhsRunning(bs, q) ? double(z32[id]) / bs->vscale[q] : 0.0;
    }
}

// ---- the C ABI's dense vectors (nrhs consecutive vectors of 3 NX NY NZ values, node i + NX (j + NY k))
// <-> the block layout over pitched nodes; 32 consecutive dense DOFs x RB right-hand sides per
// thread block through shared memory, so both sides are read and written contiguously. Right-hand
// sides q >= nrhs read as 0 and are not written back. scale (optional, per right-hand side)
// multiplies the values on the way.
template <int RB>
__global__ void __launch_bounds__(256) kb_pack(double* __restrict__ dense, int nrhs, long long nDense, double* __restrict__ blk, int NX,
                                               int NY, int PX, int toBlock, const double* __restrict__ scale) {
    __shared__ double tile[RB][33];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
    for (long long e0 = (long long)blockIdx.x * 32; e0 < nDense; e0 += (long long)gridDim.x * 32) {
        const long long e = e0 + tx;
        if (toBlock) {
            for (int q = ty; q < RB; q += 8) tile[q][tx] = (q < nrhs && e < nDense) ? dense[(long long)q * nDense + e] : 0.0;
            __syncthreads();
            // write: for each of the 32 DOFs, the RB values of its right-hand sides
            for (int w = threadIdx.x; w < 32 * RB; w += 256) {
                const int de = w / RB, q = w - de * RB;
                const long long ee = e0 + de;
                if (ee < nDense) {
                    const long long nd = ee / 3, row = nd / NX;
                    const long long pn = (nd - row * NX) + (long long)PX * row;
                    blk[(3 * pn + (ee - 3 * nd)) * RB + q] = scale ? tile[q][de] * scale[q] : tile[q][de];
                }
            }
        } else {
            for (int w = threadIdx.x; w < 32 * RB; w += 256) {
                const int de = w / RB, q = w - de * RB;
                const long long ee = e0 + de;
                double v = 0.0;
                if (ee < nDense) {
                    const long long nd = ee / 3, row = nd / NX;
                    const long long pn = (nd - row * NX) + (long long)PX * row;
                    v = blk[(3 * pn + (ee - 3 * nd)) * RB + q];
                    if (scale) v *= scale[q];
                }
                tile[q][de] = v;
            }
            __syncthreads();
            for (int q = ty; q < nrhs && q < RB; q += 8)
                if (e < nDense) dense[(long long)q * nDense + e] = tile[q][tx];
        }
        __syncthreads();
    }
    (void)NY;
}

// held DOFs of every right-hand side set to 0 over all pitched nodes (a warm start's held values)
template <int RB>
__global__ void kb_mask_fixed(long long nNodes, const uint8_t* __restrict__ nmask, double* __restrict__ x) {
    const long long total = nNodes * 3 * RB;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const long long dof = e / RB, n = dof / 3;
        if (fixedDof(nmask[n], int(dof - 3 * n))) x[e] = 0.0;
    }
}

// right-hand side q of a block vector set to 0
template <int RB>
__global__ void kb_zero_rhs(long long nNodes, double* __restrict__ x, int q) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nNodes * 3; e += (long long)gridDim.x * blockDim.x) x[e * RB + q] = 0.0;
}

}  // namespace dev
}  // namespace psfea
