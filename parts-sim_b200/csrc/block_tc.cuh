// Block operator on the tensor cores for the finest level (all voxels s * Kb). Included by
// solver.cu only.
//
// The 32-wide block's FP32 product is FMA-bound on the CUDA cores (576 FMAs per node and right-hand
// side). Here it runs element by element on the tensor pipe: for each solid voxel v,
// Y_v (24 x 32) = Kb (24 x 24) * U_v (24 x 32), U_v the voxel's 24 corner values of the 32
// right-hand sides less the voxel's corner-0 value (per component and right-hand side; Kb
// annihilates translations, so Y is unchanged while the TF32 rounding scales with the local
// variation), as warp-level mma.sync m16n8k8 TF32 products (Kb in two 16-row tiles, 24 rows used;
// three 8-wide k-steps; four 8-column right-hand-side tiles) with Kb's fragments held in registers.
// One CTA owns an 8 x 4 x 4 node tile and takes the solid voxels of its 9 x 5 x 5 footprint; each
// warp scatters s_v Y_v to the owned corners' accumulators in shared memory. Voxels are taken colour
// by colour (the parity of the voxel index per axis): voxels of one colour share no node, so the
// adds of one colour never collide, and every node's sum runs in the fixed colour order
// (deterministic). The tile kernel's epilogues (APPLY / CHEB / RESID) follow.
#pragma once

#include "block_kernels.cuh"

namespace psfea {
namespace dev {

constexpr int BT_X = 8, BT_Y = 4, BT_Z = 4, BT_NODES = BT_X * BT_Y * BT_Z, BT_THREADS = 256;
constexpr int BT_VX = BT_X + 1, BT_VY = BT_Y + 1, BT_VZ = BT_Z + 1, BT_VOX = BT_VX * BT_VY * BT_VZ;  // 225
constexpr size_t btSmemBytes() { return size_t(BT_NODES) * 3 * 32 * 4 + size_t(BT_VOX) * 4 + 8 * 64 * 2 + 64; }

__device__ __forceinline__ uint32_t toTf32(float v) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(v));
    return r;
}

__device__ __forceinline__ void mmaTf32(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

template <int MODE>
__global__ void __launch_bounds__(BT_THREADS, 2)
    kb_tc(LevelView L, Coefs<float> C, const uint32_t* __restrict__ tiles, const float* __restrict__ x, float* __restrict__ y,
          const float* __restrict__ r, float* __restrict__ d, float c1, float c2, int raw, Ctl ctl) {
    if (skipped(ctl)) return;
    constexpr int RB = 32;
    extern __shared__ __align__(16) unsigned char btRaw[];
    float* acc = reinterpret_cast<float*>(btRaw);                                  // [node][3][32]
    uint32_t* ws = reinterpret_cast<uint32_t*>(acc + BT_NODES * 3 * RB);          // footprint words
    int16_t* lists = reinterpret_cast<int16_t*>(ws + BT_VOX);                     // [colour][64]
    int* counts = reinterpret_cast<int*>(lists + 8 * 64);                         // [8]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, t = lane & 3;
    const uint32_t tw = tiles[blockIdx.x];
    const int i0 = int(tw & 2047u) * BT_X, j0 = int((tw >> 11) & 2047u) * BT_Y, k0 = int(tw >> 22) * BT_Z;
    const long long NXp = L.PX, NXY = (long long)L.PX * L.NY;

    for (int e = tid; e < BT_NODES * 3 * RB; e += BT_THREADS) acc[e] = 0.f;
    if (tid < 8) counts[tid] = 0;
    __syncthreads();
    for (int e = tid; e < BT_VOX; e += BT_THREADS) {
        const int vx = e % BT_VX, vy = (e / BT_VX) % BT_VY, vz = e / (BT_VX * BT_VY);
        const int gi = i0 - 1 + vx, gj = j0 - 1 + vy, gk = k0 - 1 + vz;
        const uint32_t w = (gi >= 0 && gj >= 0 && gk >= 0 && gi < L.nx && gj < L.ny && gk < L.nz) ? __ldg(L.word + L.wi(gi, gj, gk)) : 0u;
        ws[e] = w;
        if (w) {
            const int col = (gi & 1) | ((gj & 1) << 1) | ((gk & 1) << 2);
            const int at = atomicAdd(&counts[col], 1);
            lists[col * 64 + at] = int16_t(e);
        }
    }
    // Kb's A fragments (rows m = 3 a + c of the output, 24 used of 32; columns k = 3 b + c')
    uint32_t A[2][3][4];
#pragma unroll
    for (int mt = 0; mt < 2; mt++)
#pragma unroll
        for (int kk = 0; kk < 3; kk++) {
            const int r0 = 16 * mt + g, r1 = r0 + 8, c0 = 8 * kk + t, c1i = c0 + 4;
            A[mt][kk][0] = r0 < 24 ? toTf32(C.Kb[r0 * 24 + c0]) : 0u;
            A[mt][kk][1] = r1 < 24 ? toTf32(C.Kb[r1 * 24 + c0]) : 0u;
            A[mt][kk][2] = r0 < 24 ? toTf32(C.Kb[r0 * 24 + c1i]) : 0u;
            A[mt][kk][3] = r1 < 24 ? toTf32(C.Kb[r1 * 24 + c1i]) : 0u;
        }
    __syncthreads();
    for (int col = 0; col < 8; col++) {
        const int cnt = counts[col];
        for (int q = warp; q < cnt; q += BT_THREADS / 32) {
            const int v = lists[col * 64 + q];
            const int vx = v % BT_VX, vy = (v / BT_VX) % BT_VY, vz = v / (BT_VX * BT_VY);
            const int gi = i0 - 1 + vx, gj = j0 - 1 + vy, gk = k0 - 1 + vz;
            const long long n0 = gi + NXp * gj + NXY * gk;  // corner 0 of the voxel (always inside the grid)
            // U fragments: B[k][n] = x(corner k / 3, comp k % 3) of right-hand side n, less corner 0's value
            float base[3][4];
#pragma unroll
            for (int c = 0; c < 3; c++)
#pragma unroll
                for (int nt = 0; nt < 4; nt++) base[c][nt] = __ldg(x + (3 * n0 + c) * RB + 8 * nt + g);
            float D[2][4][4];
#pragma unroll
            for (int mt = 0; mt < 2; mt++)
#pragma unroll
                for (int nt = 0; nt < 4; nt++) D[mt][nt][0] = D[mt][nt][1] = D[mt][nt][2] = D[mt][nt][3] = 0.f;
#pragma unroll
            for (int kk = 0; kk < 3; kk++) {
                const int ka = 8 * kk + t, kb = ka + 4;  // this lane's two k rows
                const int ba = ka / 3, ca = ka % 3, bb = kb / 3, cb = kb % 3;
                const int bxa = (ba == 1 || ba == 2 || ba == 5 || ba == 6), bya = (ba == 2 || ba == 3 || ba == 6 || ba == 7), bza = ba >> 2;
                const int bxb = (bb == 1 || bb == 2 || bb == 5 || bb == 6), byb = (bb == 2 || bb == 3 || bb == 6 || bb == 7), bzb = bb >> 2;
                const float* xa = x + (3 * (n0 + bxa + NXp * bya + NXY * bza) + ca) * RB + g;
                const float* xb = x + (3 * (n0 + bxb + NXp * byb + NXY * bzb) + cb) * RB + g;
#pragma unroll
                for (int nt = 0; nt < 4; nt++) {
                    const uint32_t b0 = toTf32(__ldg(xa + 8 * nt) - base[ca][nt]);
                    const uint32_t b1 = toTf32(__ldg(xb + 8 * nt) - base[cb][nt]);
#pragma unroll
                    for (int mt = 0; mt < 2; mt++) mmaTf32(D[mt][nt], A[mt][kk], b0, b1);
                }
            }
            // scatter s Y to the owned corners: D[mt][nt] holds rows 16 mt + g (+8), columns 8 nt + 2 t (+1)
            const float s = __uint_as_float(ws[v]);
#pragma unroll
            for (int mt = 0; mt < 2; mt++)
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int m = 16 * mt + g + 8 * h;
                    if (m >= 24) continue;
                    const int a = m / 3, c = m - 3 * a;
                    const int bx = (a == 1 || a == 2 || a == 5 || a == 6), by = (a == 2 || a == 3 || a == 6 || a == 7), bz = a >> 2;
                    const int cx = vx - 1 + bx, cy = vy - 1 + by, cz = vz - 1 + bz;  // owned node coordinates
                    if (cx < 0 || cy < 0 || cz < 0 || cx >= BT_X || cy >= BT_Y || cz >= BT_Z) continue;
                    float* o = acc + ((cx + BT_X * (cy + BT_Y * cz)) * 3 + c) * RB;
#pragma unroll
                    for (int nt = 0; nt < 4; nt++) {
                        o[8 * nt + 2 * t] += s * D[mt][nt][2 * h];
                        o[8 * nt + 2 * t + 1] += s * D[mt][nt][2 * h + 1];
                    }
                }
        }
        __syncthreads();
    }
    // epilogue over the owned nodes, one right-hand side per lane
    for (int e = tid; e < BT_NODES * 3 * RB; e += BT_THREADS) {
        const int nl = e / (3 * RB), rem = e - nl * 3 * RB, c = rem / RB, qq = rem - c * RB;
        const int cx = nl % BT_X, cy = (nl / BT_X) % BT_Y, cz = nl / (BT_X * BT_Y);
        const int gi = i0 + cx, gj = j0 + cy, gk = k0 + cz;
        if (gi >= L.PX || gj >= L.NY || gk >= L.NZ) continue;
        const long long n = gi + NXp * gj + NXY * gk;
        const uint8_t mask = __ldg(L.nmask + n);
        if (!(mask & NM_ACTIVE)) continue;  // inactive nodes stay 0 in every block vector
        const long long id = (3 * n + c) * RB + qq;
        const bool fx = fixedDof(mask, c);
        float k = acc[e];
        if (L.dadd32) k += L.dadd32[3 * n + c] * x[id];
        if constexpr (MODE == BOP_APPLY) {
            y[id] = (!raw && fx) ? 0.f : k;
        } else if constexpr (MODE == BOP_RESID) {
            y[id] = fx ? 0.f : r[id] - k;
        } else {
            if (fx) {
                d[id] = 0.f;
                y[id] = 0.f;
            } else {
                const float dn = c1 * d[id] + c2 * __ldg(L.invD + 3 * n + c) * (r[id] - k);
                d[id] = dn;
                y[id] = x[id] + dn;
            }
        }
    }
}

}  // namespace dev
}  // namespace psfea
