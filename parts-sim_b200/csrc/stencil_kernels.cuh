// Assembled stencils of the Galerkin levels. Included by solver.cu only.
//
// Below the finest level the operator's element matrices are Galerkin products (an own matrix per
// voxel, shared by classes on lattices), and a node that is not uniform takes the per-voxel gather:
// the rows of its corner in each of its up to 8 voxels, 576 multiply-adds against 24 corner values
// each, through the class matrices (voxel_fea.cpp:451-486 computes the same sums). Here each such
// node instead keeps its assembled row: the 27 3x3 blocks coupling it to its neighbours, summed once
// at setup over the voxels the two nodes share. A pass then streams 243 coefficients per node
// (coalesced: 16-byte chunks, chunk-major over the node list) and does 243 multiply-adds; the
// gather of the 27 neighbours' values is unchanged. The sums run in another order than the
// per-voxel gather (FP32 rounding differs; the stored blocks are the exact sums of the same FP32
// matrices).
#pragma once

#include "kernels.cuh"

#include <type_traits>

namespace psfea {
namespace dev {

__device__ __forceinline__ void stStn(float* p, float v, float) { *p = v; }
__device__ __forceinline__ void stStn(double* p, double v, float) { *p = v; }
__device__ __forceinline__ void stStn(__half* p, float v, float inv) { *p = __float2half_rn(v * inv); }

// one thread per (listed node, neighbour o): block (n, n + o), rows of n's corner and columns of the
// neighbour's corner in each voxel holding both (s Kb for a uniformly scaled voxel, its own matrix
// otherwise); the diagonal shift joins the centre block. Sums in CT (FP32, or FP64 for the block
// path's FP64 product), stored as floats (4-value chunks), doubles (2-value chunks) or halves
// times inv (8-value chunks).
// NODE_MAJOR: the block path's paired layout instead (row t at t * STN_ROW, block_kernels.cuh).
template <class ST, class CT = float, bool NODE_MAJOR = false>
__global__ void k_stn_build(LevelView L, Coefs<CT> C, const int* __restrict__ list, int count, ST* __restrict__ stn, float inv) {
    constexpr int CW = 16 / int(sizeof(ST));
    const long long total = (long long)count * 27;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const int t = int(e % count), m = int(e / count);
        const long long n = list[t];
        int i, j, k;
        nodeCoords(L, n, i, j, k);
        const int ox = m % 3 - 1, oy = (m / 3) % 3 - 1, oz = m / 9 - 1;
        CT blk[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int v = 0; v < 8; v++) {
            const int di = v & 1, dj = (v >> 1) & 1, dk = v >> 2;
            // the voxel at offset (di - 1, dj - 1, dk - 1) holds the neighbour when o - d + 1 is 0 or 1 per axis
            const int bx = ox - di + 1, by = oy - dj + 1, bz = oz - dk + 1;
            if (bx < 0 || bx > 1 || by < 0 || by > 1 || bz < 0 || bz > 1) continue;
            const int ei = i - 1 + di, ej = j - 1 + dj, ek = k - 1 + dk;
            if (ei < 0 || ej < 0 || ek < 0 || ei >= L.nx || ej >= L.ny || ek >= L.nz) continue;
            const uint32_t w = L.word[L.wi(ei, ej, ek)];
            if (!w) continue;
            const int a = cornerOf(1 - di, 1 - dj, 1 - dk), b = cornerOf(bx, by, bz);
            if (!(w & OWN_BIT)) {
                const CT s = CT(__uint_as_float(w));
                for (int p = 0; p < 3; p++)
                    for (int q = 0; q < 3; q++) blk[3 * p + q] += s * C.Kb[(3 * a + p) * 24 + 3 * b + q];
            } else {
                const float* M = L.own + (long long)(w & ~OWN_BIT) * 576;
                for (int p = 0; p < 3; p++)
                    for (int q = 0; q < 3; q++) blk[3 * p + q] += CT(M[(3 * a + p) * 24 + 3 * b + q]);
            }
        }
        if (m == 13 && L.dadd32)
            for (int p = 0; p < 3; p++) blk[4 * p] += sizeof(CT) == 8 ? CT(L.dadd[3 * n + p]) : CT(L.dadd32[3 * n + p]);
        for (int c = 0; c < 9; c++)
            stStn(stn + (NODE_MAJOR ? (long long)t * STN_ROW + stnPairAt(m, c / 3, c % 3) : stnAt<CW>(9 * m + c, t, count)), blk[c], inv);
    }
}

// One FP32 pass (APPLY / CHEB / RESID, the epilogues of k_list) over the listed nodes of a level
// with their assembled stencils: ST = float, or __half times the level's power-of-two scale ss.
// V = __half: the FP16 coarse-level vectors (rho and c2 as in k_list). Nodes off the list are not
// written. A thread may carry NPT nodes (list entries g, g + T, ... for T threads in the grid)
// through the same unrolled sweep so that their loads overlap; measured on the B200, two nodes a
// thread (80-90 registers, half the resident warps) made the gyroid and SIMP solves 10-14 %
// slower than one, which the passes use.
template <int MODE, class ST, class V = float, int NPT = 1>
__global__ void __launch_bounds__(256) k_stn(LevelView L, const int* __restrict__ list, int count, const ST* __restrict__ stn, float ss,
                                             const V* __restrict__ x, V* __restrict__ y, const V* __restrict__ r, V* __restrict__ d, float c1,
                                             float c2, float rho, int raw, Ctl ctl) {
    if (skipped(ctl)) return;
    constexpr bool H = !std::is_same<V, float>::value;
    constexpr int CW = std::is_same<ST, float>::value ? 4 : 8;
    const long long NX = L.PX, NXY = (long long)L.PX * L.NY;
    const long long T = (long long)gridDim.x * blockDim.x;
    for (long long t0 = blockIdx.x * (long long)blockDim.x + threadIdx.x; t0 < count; t0 += NPT * T) {
        long long n[NPT], t[NPT];
        bool live[NPT];
        int ii[NPT], jj[NPT], kk[NPT];
        uint8_t mask[NPT];
#pragma unroll
        for (int u = 0; u < NPT; u++) {
            t[u] = t0 + u * T;
            live[u] = t[u] < count;
            if (!live[u]) t[u] = t0;  // a repeat of the first node, computed and not stored
            n[u] = list[t[u]];
            mask[u] = __ldg(L.nmask + n[u]);
            nodeCoords(L, n[u], ii[u], jj[u], kk[u]);
        }
        float a[NPT][3];
        float cf[NPT][CW];
#pragma unroll
        for (int u = 0; u < NPT; u++) a[u][0] = a[u][1] = a[u][2] = 0.f;
        int have = -1;  // the chunk in cf (known at compile time once the loops are unrolled)
#pragma unroll
        for (int m = 0; m < 27; m++) {
            const int ox = m % 3 - 1, oy = (m / 3) % 3 - 1, oz = m / 9 - 1;
            float xm[NPT][3];
#pragma unroll
            for (int u = 0; u < NPT; u++) {
                // no voxel couples the node to a neighbour outside the grid: its values read as 0
                const bool in = ii[u] + ox >= 0 && jj[u] + oy >= 0 && kk[u] + oz >= 0 && ii[u] + ox < L.NX && jj[u] + oy < L.NY &&
                                kk[u] + oz < L.NZ;
                const V* xp = x + 3 * (n[u] + ox + oy * NX + oz * NXY);
                xm[u][0] = in ? ldv<float>(xp) : 0.f;
                xm[u][1] = in ? ldv<float>(xp + 1) : 0.f;
                xm[u][2] = in ? ldv<float>(xp + 2) : 0.f;
            }
#pragma unroll
            for (int e = 0; e < 9; e++) {
                const int c = 9 * m + e;
                if (c / CW != have) {
                    have = c / CW;
#pragma unroll
                    for (int u = 0; u < NPT; u++) ldChunk(stn + ((long long)have * count + t[u]) * CW, cf[u]);
                }
#pragma unroll
                for (int u = 0; u < NPT; u++) a[u][e / 3] += cf[u][c % CW] * xm[u][e % 3];
            }
        }
        const float sc = (std::is_same<ST, float>::value ? 1.f : ss) * (H ? rho : 1.f);
#pragma unroll
        for (int u = 0; u < NPT; u++) {
            if (!live[u]) continue;
#pragma unroll
            for (int q = 0; q < 3; q++) {
                const float acc = a[u][q] * sc;
                const long long id = 3 * n[u] + q;
                const bool fx = fixedDof(mask[u], q);
                if (MODE == TOP_APPLY) {
                    stv(y + id, (!raw && fx) ? 0.f : acc);
                } else if (MODE == TOP_RESID) {
                    stv(y + id, fx ? 0.f : ldf(r + id) - acc);
                } else {
                    if (fx) {
                        stv(d + id, 0.f);
                        stv(y + id, 0.f);
                    } else {
                        const float dn = c1 * ldf(d + id) + c2 * L.invD[id] * (ldf(r + id) - acc);
                        stv(d + id, dn);
                        stv(y + id, ldf(x + id) + dn);
                    }
                }
            }
        }
    }
}

}  // namespace dev
}  // namespace psfea
