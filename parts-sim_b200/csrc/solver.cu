// Device-resident multigrid-preconditioned CG for one voxel model on one B200 (sm_100a).
//
// The solve loop never waits for the host inside an iteration: dot products finish in the last
// block of the kernel that computes them (deterministic order), which also derives alpha / beta
// and the stop decision into a device-side state record; every later kernel of the iteration reads
// that record and exits at once when the solve is over. The host replays a CUDA graph of one
// iteration in batches and reads the record back only between batches.
//
// Algorithms (rules of the reference, native/src/fea/voxel_fea.cpp):
//   operator apply ......................... :393-504
//   degree-2 Chebyshev smoother ............ :692-725
//   restriction / prolongation ............. :739-815
//   V-cycle ................................ :817-828
//   FP32 preconditioner, r scaled to O(1) .. :835-861
//   flexible PCG, Polak-Ribiere beta ....... :863-927
//   Lanczos smoother bound (LCG start) ..... :579-610
// The mixed-precision form keeps the CG in FP32 and folds its iterate into an FP64 solution with
// the FP64 defect as its new residual whenever the FP32 residual has fallen tenfold ("reliable
// updates", Sleijpen & van der Vorst 1996; the reference GPU solver does the fold on the CPU,
// native/src/gpu/gpu_fea.cpp:452-574); here it is a device kernel.
#include "solver.hpp"

#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <map>
#include <memory>
#include <tuple>
#include <type_traits>
#include <mutex>
#include <thread>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "host_util.hpp"
#include "kernels.cuh"

namespace psfea {

namespace dev {

// ---------------------------------------------------------------- control

struct SolveState {
    double bnorm, rel, tol, rz, alpha, beta, rmax, scale, peak, est, pq, foldFactor;
    double pqPart;  // the tiled product's share of p.q, completed by the boundary-node kernel
    double vscale;  // the scale the current FP32 right-hand side r32 was made with (r32 = r * vscale)
    int it, maxIter, done, status, fold, folds, first, mixed;
    int err;  // a device-side failure (ST_ERR_*): the solve is ended and reported as a CUDA error
    // iterative refinement (PS_PREC_HALF): each fold rescales the FP32 residual to max |r| = 1
    // (r32 *= rescale, due while restart is set) and restarts the FP32 recurrence (beta = 0)
    int refine, restart;
    double rescale;
};
enum { ST_RUNNING = 0, ST_CONVERGED = 1, ST_MAXITER = 2, ST_BREAKDOWN = 3 };

// a kernel runs unless *skipIf != 0 or (runIf and *runIf == 0)
struct Ctl {
    const int* skipIf;
    const int* runIf;
};
__device__ __forceinline__ bool skipped(const Ctl& c) {
    if (c.skipIf && *((volatile const int*)c.skipIf)) return true;
    if (c.runIf && !*((volatile const int*)c.runIf)) return true;
    return false;
}

__device__ __forceinline__ bool fixedDof(uint8_t mask, int d) { return (mask >> d) & 1; }

constexpr int NODE_THREADS = 128;
constexpr int VEC_THREADS = 256;

// ---------------------------------------------------------------- operator kernels

enum { OP_APPLY = 0, OP_CHEB = 1, OP_RESID = 2 };

// One pass over the level's nodes of y = K x with a per-node epilogue:
//   OP_APPLY  y = K x (held DOFs 0 unless raw)
//   OP_CHEB   d = c1 d + c2 D^-1 (r - K x); y = x + d      (Chebyshev / Jacobi step, 32-bit)
//   OP_RESID  y = r - K x
template <class T, int MODE, bool OWN16, bool DIFF = false>
__global__ void __launch_bounds__(NODE_THREADS) k_op(LevelView L, Coefs<T> C, const T* __restrict__ x, T* __restrict__ y,
                                                      const float* __restrict__ r, float* __restrict__ d, float c1, float c2, int raw,
                                                      Ctl ctl) {
    if (skipped(ctl)) return;
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < L.nNodes; n += (long long)gridDim.x * blockDim.x) {
        const uint8_t mask = __ldg(L.nmask + n);
        int i, j, k;
        nodeCoords(L, n, i, j, k);
        T acc[3];
        applyAt<T, OWN16, DIFF>(L, C, x, i, j, k, n, mask, acc, L.PX, n);
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const long long id = 3 * n + q;
            const bool fx = fixedDof(mask, q);
            if (MODE == OP_APPLY) {
                y[id] = (!raw && fx) ? T(0) : acc[q];
            } else if (MODE == OP_RESID) {
                y[id] = fx ? T(0) : T(r[id]) - acc[q];
            } else {
                if (fx) {
                    d[id] = 0.f;
                    y[id] = T(0);
                } else {
                    const float dn = c1 * d[id] + c2 * L.invD[id] * (r[id] - float(acc[q]));
                    d[id] = dn;
                    y[id] = x[id] + T(dn);
                }
            }
        }
    }
}

// q = K p on the finest level with the CG step length: alpha = rz / (p . q) (FP64 accumulation);
// p.q <= 0 ends the solve as a breakdown (voxel_fea.cpp:902-905)
template <class T, bool OWN16>
__global__ void __launch_bounds__(NODE_THREADS) k_apply_alpha(LevelView L, Coefs<T> C, const T* __restrict__ p, T* __restrict__ q,
                                                              SolveState* st, double* partials, unsigned* ticket, Ctl ctl) {
    if (skipped(ctl)) return;
    double v[1] = {0.0};
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < L.nNodes; n += (long long)gridDim.x * blockDim.x) {
        const uint8_t mask = __ldg(L.nmask + n);
        int i, j, k;
        nodeCoords(L, n, i, j, k);
        T acc[3];
        applyAt<T, OWN16, (sizeof(T) == 4)>(L, C, p, i, j, k, n, mask, acc, L.PX, n);
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const T y = fixedDof(mask, c) ? T(0) : acc[c];
            q[3 * n + c] = y;
            v[0] += double(p[3 * n + c]) * double(y);
        }
    }
    double tot[1];
    if (gridReduce<1>(v, 0u, partials, ticket, tot) && threadIdx.x == 0) {
        const double pq = tot[0];
        st->pq = pq;
        if (!(pq > 0)) {
            st->status = ST_BREAKDOWN;
            if (st->mixed) st->fold = 1;  // fold what there is, then stop
            else st->done = 1;
        } else {
            st->alpha = st->rz / pq;
        }
    }
}

// ---------------------------------------------------------------- coarse-level operator kernel

// The same operator and epilogues (OP_APPLY / OP_CHEB / OP_RESID) with eight lanes per node, one
// per surrounding voxel: each lane gathers its voxel's 8 corner values and applies the 3 rows of
// its corner (Kb from shared memory, or the voxel's own matrix), and the eight partial sums meet
// by shuffles. Coarse levels have few nodes and many own matrices; spreading a node over eight
// lanes turns one thread's chain of eight dependent matrix reads into eight parallel ones.
template <class T, int MODE, bool OWN16, bool DIFF>
__global__ void __launch_bounds__(256) k_op8(LevelView L, Coefs<T> C, const T* __restrict__ x, T* __restrict__ y,
                                             const float* __restrict__ r, float* __restrict__ d, float c1, float c2, int raw, Ctl ctl) {
    if (skipped(ctl)) return;
    __shared__ T kb[576];
    for (int e = threadIdx.x; e < 576; e += blockDim.x) kb[e] = C.Kb[e];
    __syncthreads();
    const int lane = threadIdx.x & 31, v = lane & 7, group = lane >> 3;
    const int di = v & 1, dj = (v >> 1) & 1, dk = v >> 2, a = cornerOf(1 - di, 1 - dj, 1 - dk);
    const long long NX = L.PX, NXY = (long long)L.PX * L.NY;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long nb = ((long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 4; nb < L.nNodes; nb += warps * 4) {
        const long long n = nb + group;
        const bool valid = n < L.nNodes;
        const uint8_t mask = valid ? __ldg(L.nmask + n) : uint8_t(0);
        T acc[3] = {T(0), T(0), T(0)};
        if (mask & NM_ACTIVE) {
            int i, j, k;
            nodeCoords(L, n, i, j, k);
            const int ei = i - 1 + di, ej = j - 1 + dj, ek = k - 1 + dk;
            uint32_t w = 0;
            if (ei >= 0 && ej >= 0 && ek >= 0 && ei < L.nx && ej < L.ny && ek < L.nz)
                w = __ldg(L.word + L.wi(ei, ej, ek));
            if (w) {
                T own[3] = {T(0), T(0), T(0)};
                if (DIFF) {
                    own[0] = __ldg(x + 3 * n);
                    own[1] = __ldg(x + 3 * n + 1);
                    own[2] = __ldg(x + 3 * n + 2);
                }
                T xe[24];
#pragma unroll
                for (int b = 0; b < 8; b++) {
                    const int bx = (b == 1 || b == 2 || b == 5 || b == 6), by = (b == 2 || b == 3 || b == 6 || b == 7), bz = b >> 2;
                    const T* xp = x + 3 * (n + (di + bx - 1) + (dj + by - 1) * NX + (dk + bz - 1) * NXY);
                    xe[3 * b] = __ldg(xp) - own[0];
                    xe[3 * b + 1] = __ldg(xp + 1) - own[1];
                    xe[3 * b + 2] = __ldg(xp + 2) - own[2];
                }
                if (!(w & OWN_BIT)) {
                    const T* k0 = kb + (3 * a) * 24;
                    T t0 = 0, t1 = 0, t2 = 0;
#pragma unroll
                    for (int q = 0; q < 24; q++) {
                        t0 += k0[q] * xe[q];
                        t1 += k0[24 + q] * xe[q];
                        t2 += k0[48 + q] * xe[q];
                    }
                    const T s = T(__uint_as_float(w));
                    acc[0] = s * t0;
                    acc[1] = s * t1;
                    acc[2] = s * t2;
                } else if (OWN16) {
                    T t[3];
                    own16Rows<T>(L.own16 + (long long)(w & ~OWN_BIT) * 576 + 72 * a, xe, t);
#pragma unroll
                    for (int dd = 0; dd < 3; dd++) acc[dd] = T(L.hs) * t[dd];
                } else {
                    const float4* K4 = reinterpret_cast<const float4*>(L.own + (long long)(w & ~OWN_BIT) * 576 + 72 * a);
#pragma unroll
                    for (int dd = 0; dd < 3; dd++) {
                        T t = 0;
#pragma unroll
                        for (int q = 0; q < 6; q++) {
                            const float4 kv = __ldg(K4 + dd * 6 + q);
                            t += T(kv.x) * xe[4 * q] + T(kv.y) * xe[4 * q + 1] + T(kv.z) * xe[4 * q + 2] + T(kv.w) * xe[4 * q + 3];
                        }
                        acc[dd] = t;
                    }
                }
            }
            if (v == 0 && L.dadd) {
#pragma unroll
                for (int q = 0; q < 3; q++) acc[q] += (sizeof(T) == 8 ? T(L.dadd[3 * n + q]) : T(L.dadd32[3 * n + q])) * x[3 * n + q];
            }
        }
#pragma unroll
        for (int o = 1; o < 8; o <<= 1)
#pragma unroll
            for (int q = 0; q < 3; q++) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
        if (valid && v < 3) {
            const int q = v;
            const long long id = 3 * n + q;
            const bool fx = fixedDof(mask, q);
            const T kx = q == 0 ? acc[0] : (q == 1 ? acc[1] : acc[2]);
            if (MODE == OP_APPLY) {
                y[id] = (!raw && fx) ? T(0) : kx;
            } else if (MODE == OP_RESID) {
                y[id] = fx ? T(0) : T(r[id]) - kx;
            } else {
                if (fx) {
                    d[id] = 0.f;
                    y[id] = T(0);
                } else {
                    const float dn = c1 * d[id] + c2 * L.invD[id] * (r[id] - float(kx));
                    d[id] = dn;
                    y[id] = x[id] + T(dn);
                }
            }
        }
    }
}

// ---------------------------------------------------------------- tiled operator kernel

// The level's operator over its active tiles with a per-node epilogue:
//   TOP_APPLY  y = K x (held DOFs 0 unless raw)
//   TOP_CHEB   d = c1 d + c2 D^-1 (r - K x); y = x + d      (Chebyshev / Jacobi step, 32-bit)
//   TOP_RESID  y = r - K x
//   TOP_DOT    y = K x (held 0) and the CG step alpha = rz / (x . y); x . y <= 0 is a breakdown
//              (voxel_fea.cpp:902-905)
// A staging barrier that never completes (it cannot in a correct launch) is given up after a
// bounded wait: the CTA records ST_ERR_STAGING in st->err and ends the solve.
constexpr unsigned TILE_WAIT_POLLS = 1u << 22;
constexpr int ST_ERR_STAGING = 1, ST_ERR_ALIGN = 2;

// the epilogue of tile node (cx, cy, cz) with its K x: results into the output tile (and d)
template <class T, int MODE>
__device__ __forceinline__ void tileFinish(const LevelView& L, const TileIO<T>& io, int i0, int j0, int k0, int cx, int cy, int cz, uint8_t mask,
                                           const T kxIn[3], const float* is, const T* xs, T* ys, float* rs, float* ds, double& dot) {
    const int base = (cz * TY + cy) * TROW + 3 * cx, xb = xOff(cx, cy, cz);
    const bool act = mask & NM_ACTIVE;
#pragma unroll
    for (int comp = 0; comp < 3; comp++) {
        const int e = base + comp;
        const bool fx = fixedDof(mask, comp);
        const T xv = xs[xb + comp];
        T kx = act ? kxIn[comp] : T(0);
        if (act && L.dadd) {
            const long long id = 3 * ((long long)(i0 + cx) + (long long)L.PX * ((j0 + cy) + (long long)L.NY * (k0 + cz))) + comp;
            kx += (sizeof(T) == 8 ? T(L.dadd[id]) : T(L.dadd32[id])) * xv;
        }
        if constexpr (MODE == TOP_APPLY) {
            ys[e] = (!io.raw && fx) ? T(0) : kx;
        } else if constexpr (MODE == TOP_DOT) {
            const T yv = fx ? T(0) : kx;
            ys[e] = yv;
            dot += double(xv) * double(yv);
        } else if constexpr (MODE == TOP_RESID) {
            rs[e] = fx ? 0.f : rs[e] - float(kx);
        } else {
            if (fx) {
                ds[e] = 0.f;
                rs[e] = 0.f;
            } else {
                const float dn = io.c1 * ds[e] + io.c2 * is[e] * (rs[e] - float(kx));
                ds[e] = dn;
                rs[e] = float(xv) + dn;
            }
        }
    }
}

// resident CTAs per SM the register budget is cut for (32-bit / 64-bit values)
#ifndef PSFEA_TILE_CTAS32
#define PSFEA_TILE_CTAS32 3
#endif
#ifndef PSFEA_TILE_CTAS64
#define PSFEA_TILE_CTAS64 2
#endif

template <class T> struct CoefsFor { using type = Coefs<T>; };
template <> struct CoefsFor<float> { using type = Coefs32; };

template <class T, int MODE, bool OWN16, bool DIFF, bool INNER = (sizeof(T) == 4)>
__global__ void __launch_bounds__(TILE_THREADS, sizeof(T) == 8 ? PSFEA_TILE_CTAS64 : PSFEA_TILE_CTAS32)
    k_tile(LevelView L, typename CoefsFor<T>::type C, const uint32_t* __restrict__ tiles, const __grid_constant__ TileMaps maps, TileIO<T> io, SolveState* st,
           double* partials, unsigned* ticket, Ctl ctl) {
    if (skipped(ctl)) return;
    using Op = TileOp<T, OWN16, DIFF>;
    extern __shared__ __align__(128) unsigned char smem[];
    if (smemAddr(smem) & 127u) {  // the layout's TMA alignment (never expected to fail)
        if (threadIdx.x == 0) {
            atomicExch(&st->err, ST_ERR_ALIGN);
            st->done = 1;
        }
        return;
    }
    T* xs = reinterpret_cast<T*>(smem);
    uint32_t* vs = reinterpret_cast<uint32_t*>(smem + tileOffW<T>());
    T* ys = reinterpret_cast<T*>(smem + tileOffY<T>());        // y tile (APPLY / DOT)
    float* rs = reinterpret_cast<float*>(smem + tileOffY<T>()); // r tile, then y in place (CHEB / RESID)
    float* ds = reinterpret_cast<float*>(smem + tileOffD<T, MODE>());
    const float* is = reinterpret_cast<const float*>(smem + tileOffI<T, MODE>());
    uint8_t* ms = smem + tileOffM<T, MODE>();
    uint16_t* blist = reinterpret_cast<uint16_t*>(smem + tileOffB<T, MODE, INNER>());
    int* wsum = reinterpret_cast<int*>(blist + TILE_NODES);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + tileOffBar<T, MODE, INNER>());  // [0] x and words, [1] r and d
    const uint32_t tw = tiles[blockIdx.x];
    const int i0 = int(tw & 2047u) * TX, j0 = int((tw >> 11) & 2047u) * TY, k0 = int(tw >> 22) * TZ;
    const int tid = threadIdx.x, cx = tid & 31, cy = tid >> 5;
    const long long PXY = (long long)L.PX * L.NY;

    // stage: one thread issues every copy, on two barriers
    if (tid == 0) {
        mbarInit(bar, 1);
        mbarInit(bar + 1, 1);
        mbarExpectTx(bar, tileStage0Bytes<T>());
        tmaLoad3d(xs, &maps.x, 3 * (i0 - XLEFT), j0 - 1, k0 - 1, bar);
        tmaLoad3d(vs, &maps.w, i0 - XLEFT, j0 - 1, k0 - 1, bar);
        if (tileHasR(MODE)) {
            mbarExpectTx(bar + 1, tileStage1Bytes<MODE>());
            tmaLoad3d(rs, &maps.r, 3 * i0, j0, k0, bar + 1);
            if (tileHasD(MODE)) {
                tmaLoad3d(ds, &maps.d, 3 * i0, j0, k0, bar + 1);
                tmaLoad3d(const_cast<float*>(is), &maps.inv, 3 * i0, j0, k0, bar + 1);
            }
        }
    }
    // the column's node masks (padding nodes i >= NX hold 7: inactive, all held) meanwhile
    const int i = i0 + cx, j = j0 + cy;
    const bool col = i < L.PX && j < L.NY;
    uint8_t mk[TZ];
    bool anyUniform = false;
    unsigned bmask = 0;  // the column's boundary nodes (active, not uniform)
#pragma unroll
    for (int z = 0; z < TZ; z++) {
        const int k = k0 + z;
        mk[z] = (col && k < L.NZ) ? __ldg(L.nmask + i + (long long)L.PX * j + PXY * k) : uint8_t(0);
        if (INNER) ms[(z * TY + cy) * TX + cx] = mk[z];
        anyUniform = anyUniform || (mk[z] & NM_UNIFORM);
        if ((mk[z] & NM_ACTIVE) && !(mk[z] & NM_UNIFORM)) bmask |= 1u << z;
    }
    int total = 0;
    if constexpr (INNER) {
        // the boundary nodes compacted in a fixed order (thread order, then z) while the copies land
        const int cnt = __popc(bmask);
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (cx >= o) incl += v;
        }
        if (cx == 31) wsum[cy] = incl;
        if (tid == 0) wsum[TILE_THREADS / 32] = 0;  // the counter of handed-out boundary chunks
        __syncthreads();
        int off = incl - cnt;
#pragma unroll
        for (int w = 0; w < TILE_THREADS / 32; w++) {
            const int c = wsum[w];
            off += (w < cy) ? c : 0;
            total += c;
        }
        for (unsigned b = bmask; b; b &= b - 1) blist[off++] = uint16_t((tid << 4) | (__ffs(b) - 1));
    }
    __syncthreads();  // barriers initialised; masks and the boundary list in place
    // each warp goes on as soon as its own wait ends; the outcome is combined before the stores
    bool ok = mbarWait(bar, TILE_WAIT_POLLS);
    double dot = 0.0;
    // pass 1: the thread's column, all four nodes from one sweep of the planes (uniform nodes)
    T acc[TZ][3];
    if (ok && anyUniform) {
        if constexpr (sizeof(T) == 4) Op::column2(C, xs, cx, cy, acc);
        else Op::column(C, xs, cx, cy, acc);
    }
    if (tileHasR(MODE)) ok = ok && mbarWait(bar + 1, TILE_WAIT_POLLS);
    if (ok) {
        // epilogue of the column's nodes except the boundary ones. An inactive node (all its DOFs
        // held; r, d and x are 0 there) gives y = 0: with r staged in place of the output
        // (smoother, residual) its slots already hold that, a separate output tile gets zeros
#pragma unroll
        for (int z = 0; z < TZ; z++) {
            if ((bmask >> z) & 1u) continue;
            if (!(mk[z] & NM_ACTIVE)) {
                if (!tileHasR(MODE)) {  // a separate output tile: its slots are zeros
                    T* yn = ys + (z * TY + cy) * TROW + 3 * cx;
                    yn[0] = yn[1] = yn[2] = T(0);
                }
                continue;
            }
            T kx[3] = {T(0), T(0), T(0)};
            if (mk[z] & NM_UNIFORM) {
                const T s = T(__uint_as_float(vs[vOff(cx, cy, z)]));
                kx[0] = s * acc[z][0];
                kx[1] = s * acc[z][1];
                kx[2] = s * acc[z][2];
            }
            tileFinish<T, MODE>(L, io, i0, j0, k0, cx, cy, z, mk[z], kx, is, xs, ys, rs, ds, dot);
        }
    }
    if constexpr (INNER) {
        // pass 2: the listed nodes in chunks of 32 to whichever warp is free first, one thread a node
        // (per-voxel gather); a node's result does not depend on the warp that computes it, and its
        // share of x.y is added below by the thread owning its column, in a fixed order
        for (;;) {
            int c = 0;
            if (cx == 0) c = atomicAdd(&wsum[TILE_THREADS / 32], 32);
            c = __shfl_sync(0xffffffffu, c, 0);
            if (c >= total) break;
            const int q = c + cx;
            if (ok && q < total) {
                const int e = blist[q], bt = e >> 4, bz = e & 15, bx = bt & 31, by = bt >> 5;
                T own[3] = {T(0), T(0), T(0)};
                if (DIFF) {
                    const T* xn = xs + xOff(bx, by, bz);
                    own[0] = xn[0]; own[1] = xn[1]; own[2] = xn[2];
                }
                T a[3];
                Op::general(L, C, xs, vs, bx, by, bz, a, own);
                double unused = 0.0;
                tileFinish<T, MODE>(L, io, i0, j0, k0, bx, by, bz, ms[(bz * TY + by) * TX + bx], a, is, xs, ys, rs, ds, unused);
            }
        }
    }
    // results out
    fenceAsyncShared();
    const bool staged = __syncthreads_and(ok) != 0;
    if (INNER && MODE == TOP_DOT && staged) {
        // the column's boundary nodes' share of x.y, from the y tile
#pragma unroll
        for (int z = 0; z < TZ; z++) {
            if (!((bmask >> z) & 1u)) continue;
            const T* xn = xs + xOff(cx, cy, z);
            const T* yn = ys + (z * TY + cy) * TROW + 3 * cx;
#pragma unroll
            for (int c = 0; c < 3; c++) dot += double(xn[c]) * double(yn[c]);
        }
    }
    if (staged && tid == 0) {
        if (tileHasR(MODE)) tmaStore3d(&maps.y, rs, 3 * i0, j0, k0);
        else tmaStore3d(&maps.y, ys, 3 * i0, j0, k0);
        if (tileHasD(MODE)) tmaStore3d(&maps.d, ds, 3 * i0, j0, k0);
        tmaStoreCommitWait();
    }
    if (!staged && tid == 0) {
        atomicExch(&st->err, ST_ERR_STAGING);
        st->done = 1;
    }
    if (MODE == TOP_DOT) {
        double vv[1] = {dot};
        double tot[1];
        if (gridReduce<1>(vv, 0u, partials, ticket, tot) && threadIdx.x == 0) {
            const double pq = tot[0];
            if (io.partial) {  // the boundary-node kernel adds its share and finishes the step
                st->pqPart = pq;
                return;
            }
            st->pq = pq;
            if (!(pq > 0)) {
                st->status = ST_BREAKDOWN;
                if (st->mixed) st->fold = 1;  // fold what there is, then stop
                else st->done = 1;
            } else {
                st->alpha = st->rz / pq;
            }
        }
    }
}

// The boundary nodes of a tiled level (active, not uniform: next to an empty voxel, a voxel of
// another scale or an own matrix) from their list, one thread each, with the per-voxel gather and
// the tiled kernel's epilogues (TOP_*); runs after the tiled kernel on the same vectors and
// overwrites the boundary nodes' output slots. TOP_DOT adds its p.q share to the tiled one
// (fixed order: tiles, then boundary nodes) and takes the CG step.
template <class T, int MODE, bool OWN16, bool DIFF>
__global__ void __launch_bounds__(NODE_THREADS) k_bnd(LevelView L, Coefs<T> C, const int* __restrict__ list, int count, const T* __restrict__ x,
                                                      T* __restrict__ y, const float* __restrict__ r, float* __restrict__ d, float c1, float c2,
                                                      int raw, SolveState* st, double* partials, unsigned* ticket, Ctl ctl) {
    if (skipped(ctl)) return;
    double v[1] = {0.0};
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < count; t += (long long)gridDim.x * blockDim.x) {
        const long long n = list[t];
        const uint8_t mask = __ldg(L.nmask + n);
        int i, j, k;
        nodeCoords(L, n, i, j, k);
        T acc[3];
        applyAt<T, OWN16, DIFF>(L, C, x, i, j, k, n, mask, acc, L.PX, n);
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const long long id = 3 * n + q;
            const bool fx = fixedDof(mask, q);
            if (MODE == TOP_APPLY) {
                y[id] = (!raw && fx) ? T(0) : acc[q];
            } else if (MODE == TOP_DOT) {
                const T yv = fx ? T(0) : acc[q];
                y[id] = yv;
                v[0] += double(x[id]) * double(yv);
            } else if (MODE == TOP_RESID) {
                y[id] = fx ? T(0) : T(r[id]) - acc[q];
            } else {
                if (fx) {
                    d[id] = 0.f;
                    y[id] = T(0);
                } else {
                    const float dn = c1 * d[id] + c2 * L.invD[id] * (r[id] - float(acc[q]));
                    d[id] = dn;
                    y[id] = x[id] + T(dn);
                }
            }
        }
    }
    if (MODE == TOP_DOT) {
        double tot[1];
        if (gridReduce<1>(v, 0u, partials, ticket, tot) && threadIdx.x == 0) {
            const double pq = st->pqPart + tot[0];
            st->pq = pq;
            if (!(pq > 0)) {
                st->status = ST_BREAKDOWN;
                if (st->mixed) st->fold = 1;  // fold what there is, then stop
                else st->done = 1;
            } else {
                st->alpha = st->rz / pq;
            }
        }
    }
}

// ---------------------------------------------------------------- V-cycle pieces (32-bit)

// z = d = c0 D^-1 r (the first Chebyshev step from zero); V = __half: the FP16 coarse-level
// vectors, c0 carrying the level's iterate-to-residual scale
template <class V = float>
__global__ void k_cheb_first(long long nDof, const V* __restrict__ r, const float* __restrict__ invD, V* __restrict__ d, V* __restrict__ z,
                             float c0, Ctl ctl) {
    if (skipped(ctl)) return;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nDof; i += (long long)gridDim.x * blockDim.x) {
        const float v = c0 * invD[i] * ldf(r + i);
        stv(d + i, v);
        stv(z + i, v);
    }
}

// rc = P^T rf gathered per coarse node: fine 2I (weight 1) and 2I +- 1 (weight 1/2) per axis;
// held / inactive coarse DOFs 0. VF / VC: the fine / coarse storage (float, or __half for the FP16
// coarse-level vectors, whose residual scales differ by the power of two sr: rc = sr P^T rf).
template <class VF = float, class VC = float>
__global__ void k_restrict(LevelView F, LevelView C, const VF* __restrict__ rf, VC* __restrict__ rc, VC* __restrict__ dc,
                           VC* __restrict__ zc, float c0, float sr, Ctl ctl) {
    if (skipped(ctl)) return;
    const int FNX = F.NX, FNY = F.NY, FNZ = F.NZ;
    const long long FPX = F.PX, FPXY = (long long)F.PX * F.NY;
    for (long long cn = blockIdx.x * (long long)blockDim.x + threadIdx.x; cn < C.nNodes; cn += (long long)gridDim.x * blockDim.x) {
        const uint8_t mask = C.nmask[cn];
        float s0 = 0, s1 = 0, s2 = 0;
        if (mask & NM_ACTIVE) {
            int I, J, K;
            nodeCoords(C, cn, I, J, K);
            for (int dk = -1; dk <= 1; dk++) {
                const int k = 2 * K + dk;
                if (k < 0 || k >= FNZ) continue;
                const float wk = dk ? 0.5f : 1.f;
                for (int dj = -1; dj <= 1; dj++) {
                    const int j = 2 * J + dj;
                    if (j < 0 || j >= FNY) continue;
                    const float wj = (dj ? 0.5f : 1.f) * wk;
                    for (int di = -1; di <= 1; di++) {
                        const int i = 2 * I + di;
                        if (i < 0 || i >= FNX) continue;
                        const float w = (di ? 0.5f : 1.f) * wj;
                        const VF* p = rf + 3 * (i + j * FPX + k * FPXY);
                        s0 += w * ldf(p);
                        s1 += w * ldf(p + 1);
                        s2 += w * ldf(p + 2);
                    }
                }
            }
        }
        const float sv[3] = {s0, s1, s2};
        constexpr bool SCALED = !std::is_same<VC, float>::value;
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const float v = fixedDof(mask, q) ? 0.f : (SCALED ? sr * sv[q] : sv[q]);
            stv(rc + 3 * cn + q, v);
            if (dc) {  // the coarse level's first smoothing step, d = z = c0 D^-1 r
                const float dv = c0 * C.invD[3 * cn + q] * v;
                stv(dc + 3 * cn + q, dv);
                stv(zc + 3 * cn + q, dv);
            }
        }
    }
}

// zf += P zc at free fine DOFs (trilinear: coarse i/2 and, when odd, (i+1)/2, weight 1/2 each);
// VC / VF as in k_restrict, the iterate scales differing by the power of two sp: zf += sp P zc.
// list: the fine level's active nodes (inactive ones are all held and never written), or null for
// every node of the level.
template <class VC = float, class VF = float>
__global__ void k_prolong(LevelView F, int CPX, int CNY, const int* __restrict__ list, long long count, const VC* __restrict__ zc,
                          VF* __restrict__ zf, float sp, Ctl ctl) {
    if (skipped(ctl)) return;
    const long long CNX = CPX, CNXY = (long long)CPX * CNY;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < count; t += (long long)gridDim.x * blockDim.x) {
        const long long fn = list ? (long long)list[t] : t;
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
                    const VC* p = zc + 3 * ((i0 + a) + (j0 + b) * CNX + (k0 + c) * CNXY);
                    s0 += w * ldf(p);
                    s1 += w * ldf(p + 1);
                    s2 += w * ldf(p + 2);
                }
        constexpr bool SCALED = !std::is_same<VC, float>::value;
        if (SCALED) {
            s0 *= sp;
            s1 *= sp;
            s2 *= sp;
        }
        if (!fixedDof(mask, 0)) stv(zf + 3 * fn, ldf(zf + 3 * fn) + s0);
        if (!fixedDof(mask, 1)) stv(zf + 3 * fn + 1, ldf(zf + 3 * fn + 1) + s1);
        if (!fixedDof(mask, 2)) stv(zf + 3 * fn + 2, ldf(zf + 3 * fn + 2) + s2);
    }
}

// coarsest level: z = A^-1 r over the m free DOFs (FP64 dense inverse, one warp per row);
// r, z are the level's vectors (float or double), held DOFs of z are never written (stay 0)
// (zs: the FP16 coarse-level vectors' iterate-to-residual scale, a power of two; 1 otherwise)
template <class TI, class TO>
__global__ void k_coarse(int m, const int* __restrict__ dof, const double* __restrict__ Ainv, const TI* __restrict__ r, TO* __restrict__ z,
                         double zs, Ctl ctl) {
    if (skipped(ctl)) return;
    extern __shared__ double rs[];
    for (int q = threadIdx.x; q < m; q += blockDim.x) rs[q] = ldv<double>(r + dof[q]);
    __syncthreads();
    const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
    for (int row = blockIdx.x * warps + (threadIdx.x >> 5); row < m; row += gridDim.x * warps) {
        const double* a = Ainv + (size_t)row * m;
        double s = 0;
        for (int c = lane; c < m; c += 32) s += a[c] * rs[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) {
            if constexpr (std::is_same<TO, __half>::value) z[dof[row]] = __double2half(s * zs);
            else z[dof[row]] = TO(s);
        }
    }
}

// ---------------------------------------------------------------- FP64 CG vector kernels

// r = f - q at free DOFs (0 at held); bnorm = ||f_free||, rel = ||r|| / bnorm, rmax = max |r_free|
// (voxel_fea.cpp:876-886). Zero load: x = 0 and the solve is over (voxel_fea.cpp:880-884).
__global__ void k_cg_init(long long nNodes, const uint8_t* __restrict__ nmask, const double* __restrict__ f, const double* __restrict__ q,
                          double* __restrict__ r, float* __restrict__ r32, SolveState* st, double* partials, unsigned* ticket) {
    double v[3] = {0, 0, 0};
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nNodes; n += (long long)gridDim.x * blockDim.x) {
        const uint8_t mask = nmask[n];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const long long id = 3 * n + c;
            double rv = 0;
            if (!fixedDof(mask, c)) {
                const double fv = f[id];
                rv = fv - q[id];
                v[0] += fv * fv;
                v[1] += rv * rv;
                v[2] = fmax(v[2], fabs(rv));
            }
            r[id] = rv;
        }
    }
    double tot[3];
    if (gridReduce<3>(v, 4u, partials, ticket, tot) && threadIdx.x == 0) {
        st->bnorm = sqrt(tot[0]);
        st->rmax = tot[2];
        st->scale = tot[2] > 0 ? 1.0 / tot[2] : 1.0;
        st->peak = 0;
        if (st->bnorm == 0) {
            st->rel = 0;
            st->status = ST_CONVERGED;
            st->done = 2;  // 2 = zero load: the solution is zero
        } else {
            st->rel = sqrt(tot[1]) / st->bnorm;
            st->peak = st->rel;
            if (st->rel <= st->tol) {
                st->status = ST_CONVERGED;
                st->done = 1;
            } else if (st->maxIter <= 0) {
                st->status = ST_MAXITER;
                st->done = 1;
            }
        }
    }
    (void)r32;
}

// x += alpha p, r -= alpha q at free DOFs; rel = ||r|| / bnorm; stop on rel <= tol or the cap.
// Fused: the preconditioner's FP32 input r32 = r * s (s = 1 / max|r_free| of the previous iterate;
// the V-cycle is linear, so any order-one scale serves, voxel_fea.cpp:843-857) and the first
// Chebyshev step of the finest level, d = z = c0 D^-1 r32.
__global__ void k_cg_update(long long nNodes, const uint8_t* __restrict__ nmask, double* __restrict__ x, double* __restrict__ r,
                            const double* __restrict__ p, const double* __restrict__ q, float* __restrict__ r32, const float* __restrict__ invD,
                            float* __restrict__ d, float* __restrict__ z, float c0, SolveState* st, double* partials, unsigned* ticket,
                            Ctl ctl) {
    if (skipped(ctl)) return;
    const double alpha = st->alpha, s = st->scale;
    double v[2] = {0, 0};
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nNodes; n += (long long)gridDim.x * blockDim.x) {
        const uint8_t mask = nmask[n];
        if ((mask & 7) == 7) continue;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            if (fixedDof(mask, c)) continue;
            const long long id = 3 * n + c;
            x[id] += alpha * p[id];
            const double rv = r[id] - alpha * q[id];
            r[id] = rv;
            v[0] += rv * rv;
            v[1] = fmax(v[1], fabs(rv));
            if (r32) {
                const float rs = float(rv * s);
                r32[id] = rs;
                const float dv = c0 * invD[id] * rs;
                d[id] = dv;
                z[id] = dv;
            }
        }
    }
    double tot[2];
    if (gridReduce<2>(v, 2u, partials, ticket, tot) && threadIdx.x == 0) {
        st->rel = sqrt(tot[0]) / st->bnorm;
        st->vscale = s;
        st->rmax = tot[1];
        st->scale = tot[1] > 0 ? 1.0 / tot[1] : 1.0;
        st->it += 1;
        if (st->rel <= st->tol) {
            st->status = ST_CONVERGED;
            st->done = 1;
        } else if (st->it >= st->maxIter) {
            st->status = ST_MAXITER;
            st->done = 1;
        }
    }
}

// the preconditioner's input: r32 = float(r / max|r_free|) at free DOFs (voxel_fea.cpp:856-857),
// and (d non-null) the first Chebyshev step d = z = c0 D^-1 r32
__global__ void k_vc_load(long long nNodes, const uint8_t* __restrict__ nmask, const double* __restrict__ r, float* __restrict__ r32,
                          const float* __restrict__ invD, float* __restrict__ d, float* __restrict__ z, float c0, SolveState* st, Ctl ctl) {
    if (skipped(ctl)) return;
    const double s = st->scale;
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nNodes; n += (long long)gridDim.x * blockDim.x) {
        const uint8_t mask = nmask[n];
        if ((mask & 7) == 7) continue;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            if (fixedDof(mask, c)) continue;
            const long long id = 3 * n + c;
            const float rs = float(r[id] * s);
            r32[id] = rs;
            if (d) {
                const float dv = c0 * invD[id] * rs;
                d[id] = dv;
                z[id] = dv;
            }
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) st->vscale = s;
}

// z = z32 / vscale (or z64); rzNew = r.z, zq = z.q; beta = max(0, -alpha zq / rz)
// (voxel_fea.cpp:913-917); on the first pass beta = 0. Held DOFs carry zeros and are skipped.
__global__ void k_cg_dots(long long nNodes, const uint8_t* __restrict__ nmask, const double* __restrict__ r, const float* __restrict__ z32,
                          const double* __restrict__ z64, const double* __restrict__ q, SolveState* st, double* partials, unsigned* ticket,
                          Ctl ctl) {
    if (skipped(ctl)) return;
    const double inv = 1.0 / st->vscale;
    const bool first = st->first;
    double v[2] = {0, 0};
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nNodes; n += (long long)gridDim.x * blockDim.x) {
        const uint8_t mask = nmask[n];
        if ((mask & 7) == 7) continue;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            if (fixedDof(mask, c)) continue;
            const long long i = 3 * n + c;
            const double z = z64 ? z64[i] : double(z32[i]) * inv;
            v[0] += r[i] * z;
            if (!first) v[1] += z * q[i];
        }
    }
    double tot[2];
    if (gridReduce<2>(v, 0u, partials, ticket, tot) && threadIdx.x == 0) {
        st->beta = first ? 0.0 : fmax(0.0, -st->alpha * tot[1] / st->rz);
        st->rz = tot[0];
    }
}

// p = z + beta p at free DOFs
__global__ void k_cg_p(long long nNodes, const uint8_t* __restrict__ nmask, const float* __restrict__ z32, const double* __restrict__ z64,
                       double* __restrict__ p, SolveState* st, Ctl ctl) {
    if (skipped(ctl)) return;
    const double inv = 1.0 / st->vscale, beta = st->beta;
    const bool first = st->first;
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nNodes; n += (long long)gridDim.x * blockDim.x) {
        const uint8_t mask = nmask[n];
        if ((mask & 7) == 7) continue;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            if (fixedDof(mask, c)) continue;
            const long long i = 3 * n + c;
            const double z = z64 ? z64[i] : double(z32[i]) * inv;
            p[i] = first ? z : z + beta * p[i];
        }
    }
}

__global__ void k_clear_first(SolveState* st) { st->first = 0; }

// true residual after the loop: ||f - K x|| over all DOFs / bnorm (voxel_fea.cpp:921-925)
__global__ void k_final(long long nNodes, const uint8_t* __restrict__ nmask, const double* __restrict__ f, const double* __restrict__ q,
                        SolveState* st, double* partials, unsigned* ticket) {
    double v[1] = {0};
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nNodes; n += (long long)gridDim.x * blockDim.x) {
        const uint8_t mask = nmask[n];
#pragma unroll
        for (int c = 0; c < 3; c++)
            if (!fixedDof(mask, c)) {
                const double rv = f[3 * n + c] - q[3 * n + c];
                v[0] += rv * rv;
            }
    }
    double tot[1];
    if (gridReduce<1>(v, 0u, partials, ticket, tot) && threadIdx.x == 0) st->rel = st->bnorm > 0 ? sqrt(tot[0]) / st->bnorm : 0.0;
}

// ---------------------------------------------------------------- mixed precision (FP32 CG + FP64 folds)

// x32 += alpha p32, r32 -= alpha q32; est = ||r32|| / (scale * bnorm); fold when est <= tol or it has
// fallen tenfold since the last fold, or at the iteration cap
// (foldIf: the graph condition of the fold's branch, set to the decision); with the V-cycle's first
// smoothing step from zero fused in, d = z = c0 D^-1 r32 (a fold redoes it on its new r32)
__global__ void k_mx_update(long long nNodes, const uint8_t* __restrict__ nmask, float* __restrict__ x, float* __restrict__ r,
                            const float* __restrict__ p, const float* __restrict__ q, const float* __restrict__ invD, float* __restrict__ d,
                            float* __restrict__ z, float c0, SolveState* st, double* partials, unsigned* ticket,
                            cudaGraphConditionalHandle foldIf, int useIf, Ctl ctl) {
    if (skipped(ctl)) return;
    if (st->fold) {  // a breakdown in the product: fold what there is
        if (useIf && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(foldIf, 1u);
        return;
    }
    const float alpha = float(st->alpha);
    double v[1] = {0};
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nNodes; n += (long long)gridDim.x * blockDim.x) {
        const uint8_t mask = nmask[n];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            if (fixedDof(mask, c)) continue;
            const long long id = 3 * n + c;
            x[id] += alpha * p[id];
            const float rv = r[id] - alpha * q[id];
            r[id] = rv;
            v[0] += double(rv) * rv;
            const float dv = c0 * invD[id] * rv;
            d[id] = dv;
            z[id] = dv;
        }
    }
    double tot[1];
    if (gridReduce<1>(v, 0u, partials, ticket, tot) && threadIdx.x == 0) {
        st->est = sqrt(tot[0]) / st->scale / st->bnorm;
        st->it += 1;
        st->peak = fmax(st->peak, st->est);
        if (st->est <= st->tol || st->est <= st->foldFactor * st->peak || st->it >= st->maxIter || !(st->est == st->est)) st->fold = 1;
        if (useIf) cudaGraphSetConditional(foldIf, st->fold ? 1u : 0u);
    }
}

// fold part 1: u += x32 / scale, x32 = 0
__global__ void k_mx_fold1(long long nDof, double* __restrict__ u, float* __restrict__ x32, const SolveState* st, Ctl ctl) {
    if (skipped(ctl)) return;
    const double inv = 1.0 / st->scale;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nDof; i += (long long)gridDim.x * blockDim.x) {
        u[i] += double(x32[i]) * inv;
        x32[i] = 0.f;
    }
}

// fold part 2 (after q = K u in FP64): r64 = f - q, rel = ||r64|| / bnorm, r32 = float(r64 * scale);
// stop when rel <= tol, at the cap or after a breakdown
__global__ void k_mx_fold2(long long nNodes, const uint8_t* __restrict__ nmask, const double* __restrict__ f, const double* __restrict__ q,
                           float* __restrict__ r32, const float* __restrict__ invD, float* __restrict__ d, float* __restrict__ z, float c0,
                           SolveState* st, double* partials, unsigned* ticket, Ctl ctl) {
    if (skipped(ctl)) return;
    const double s = st->scale;
    double v[2] = {0, 0};
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nNodes; n += (long long)gridDim.x * blockDim.x) {
        const uint8_t mask = nmask[n];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const long long id = 3 * n + c;
            double rv = 0;
            if (!fixedDof(mask, c)) rv = f[id] - q[id];
            v[0] += rv * rv;
            v[1] = fmax(v[1], fabs(rv));
            const float rs = float(rv * s);
            r32[id] = rs;
            const float dv = c0 * invD[id] * rs;
            d[id] = dv;
            z[id] = dv;
        }
    }
    double tot[2];
    if (gridReduce<2>(v, 2u, partials, ticket, tot) && threadIdx.x == 0) {
        if (st->refine && tot[1] > 0) {
            // the next inner solve starts from the defect scaled to max |r| = 1
            st->rescale = (1.0 / tot[1]) / s;
            st->scale = 1.0 / tot[1];
            st->restart = 1;
        }
        st->rel = sqrt(tot[0]) / st->bnorm;
        st->peak = st->rel;
        st->folds += 1;
        st->fold = 0;
        if (st->status == ST_BREAKDOWN) st->done = 1;
        else if (st->rel <= st->tol) {
            st->status = ST_CONVERGED;
            st->done = 1;
        } else if (st->it >= st->maxIter || !(st->rel == st->rel)) {
            st->status = ST_MAXITER;
            st->done = 1;
        }
    }
}

// rzNew = r32.z32, zq = z32.q32 (FP64 sums); beta as in the FP64 form
// r.z and z.q over the free DOFs (node by node: the held DOFs, every DOF of an inactive node
// included, add nothing and are not read)
__global__ void k_mx_dots(long long nNodes, const uint8_t* __restrict__ nmask, const float* __restrict__ r, const float* __restrict__ z,
                          const float* __restrict__ q, SolveState* st, double* partials, unsigned* ticket, Ctl ctl) {
    if (skipped(ctl)) return;
    const bool first = st->first;
    double v[2] = {0, 0};
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nNodes; n += (long long)gridDim.x * blockDim.x) {
        const uint8_t mask = nmask[n];
        if ((mask & 7) == 7) continue;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            if (fixedDof(mask, c)) continue;
            const long long i = 3 * n + c;
            const float zi = z[i];
            v[0] += double(r[i]) * zi;
            if (!first) v[1] += double(zi) * q[i];
        }
    }
    double tot[2];
    if (gridReduce<2>(v, 0u, partials, ticket, tot) && threadIdx.x == 0) {
        st->beta = (first || st->restart) ? 0.0 : fmax(0.0, -st->alpha * tot[1] / st->rz);
        st->rz = tot[0];
        st->restart = 0;
    }
}

// after a refinement fold: r32 *= rescale and the first smoothing step again (runs while
// st->restart is set)
__global__ void k_mx_rescale(long long nDof, float* __restrict__ r32, const float* __restrict__ invD, float* __restrict__ d,
                             float* __restrict__ z, float c0, const SolveState* st, Ctl ctl) {
    if (skipped(ctl)) return;
    const float f = float(st->rescale);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nDof; i += (long long)gridDim.x * blockDim.x) {
        const float rs = r32[i] * f;
        r32[i] = rs;
        const float dv = c0 * invD[i] * rs;
        d[i] = dv;
        z[i] = dv;
    }
}

// p = z + beta p at the free DOFs; the first direction of a solve also writes 0 at every held DOF,
// which then stays 0 (the later steps skip held DOFs and inactive nodes)
__global__ void k_mx_p(long long nNodes, const uint8_t* __restrict__ nmask, const float* __restrict__ z, float* __restrict__ p,
                       const SolveState* st, Ctl ctl) {
    if (skipped(ctl)) return;
    const float beta = float(st->beta);
    const bool first = st->first;
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nNodes; n += (long long)gridDim.x * blockDim.x) {
        const uint8_t mask = nmask[n];
        if (!first && (mask & 7) == 7) continue;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const long long i = 3 * n + c;
            if (fixedDof(mask, c)) {
                if (first) p[i] = 0.f;
                continue;
            }
            p[i] = first ? z[i] : z[i] + beta * p[i];
        }
    }
}

// ---------------------------------------------------------------- misc

__global__ void k_mask_copy(long long nNodes, const uint8_t* __restrict__ nmask, const double* __restrict__ src, double* __restrict__ dst) {
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nNodes; n += (long long)gridDim.x * blockDim.x) {
        const uint8_t mask = nmask[n];
#pragma unroll
        for (int c = 0; c < 3; c++) dst[3 * n + c] = (src && !fixedDof(mask, c)) ? src[3 * n + c] : 0.0;
    }
}

// max |r| over free DOFs into st->rmax / st->scale (the preconditioner entry point)
__global__ void k_rmax(long long nNodes, const uint8_t* __restrict__ nmask, const double* __restrict__ r, SolveState* st, double* partials,
                       unsigned* ticket) {
    double v[1] = {0};
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nNodes; n += (long long)gridDim.x * blockDim.x) {
        const uint8_t mask = nmask[n];
#pragma unroll
        for (int c = 0; c < 3; c++)
            if (!fixedDof(mask, c)) v[0] = fmax(v[0], fabs(r[3 * n + c]));
    }
    double tot[1];
    if (gridReduce<1>(v, 1u, partials, ticket, tot) && threadIdx.x == 0) {
        st->rmax = tot[0];
        st->scale = tot[0] > 0 ? 1.0 / tot[0] : 1.0;
    }
}

// z = z32 * rmax on active nodes, 0 elsewhere (voxel_fea.cpp:859-860)
__global__ void k_vc_store(long long nNodes, const uint8_t* __restrict__ nmask, const float* __restrict__ z32, double* __restrict__ z,
                           const SolveState* st) {
    const double inv = 1.0 / st->vscale, rmax = st->rmax;
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nNodes; n += (long long)gridDim.x * blockDim.x) {
        const bool act = nmask[n] & NM_ACTIVE;
#pragma unroll
        for (int c = 0; c < 3; c++) z[3 * n + c] = (act && rmax > 0) ? double(z32[3 * n + c]) * inv : 0.0;
    }
}

// ---- Lanczos (FP64) for the smoother's eigenvalue bound

// v_i = LCG value i (seed 12345, s <- (1103515245 s + 12345) mod 2^31, voxel_fea.cpp:584-588),
// computed for every index at once by jumping the affine recurrence ahead i + 1 steps
__global__ void k_lz_start(LevelView L, double* __restrict__ v, double* partials, unsigned* ticket, SolveState* st) {
    double acc[1] = {0};
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < L.nNodes; n += (long long)gridDim.x * blockDim.x) {
        const uint8_t mask = L.nmask[n];
        int i, j, k;
        nodeCoords(L, n, i, j, k);
        const long long nd = i + (long long)L.NX * (j + (long long)L.NY * k);  // the reference's (dense) node index
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const unsigned long long steps = (unsigned long long)(3 * nd + c) + 1;
            // (A, B): s -> A s + B for 2^bit steps; (RA, RB) accumulated
            unsigned long long A = 1103515245ull, B = 12345ull, RA = 1, RB = 0;
            const unsigned long long M = 0x7fffffffull;
            for (unsigned long long e = steps; e; e >>= 1) {
                if (e & 1) {
                    RB = (A * RB + B) & M;
                    RA = (A * RA) & M;
                }
                B = (A * B + B) & M;
                A = (A * A) & M;
            }
            const unsigned long long s = (RA * 12345ull + RB) & M;
            const double val = fixedDof(mask, c) ? 0.0 : double(s) / 2147483647.0 - 0.5;
            v[3 * n + c] = val;
            acc[0] += val * val;
        }
    }
    double tot[1];
    if (gridReduce<1>(acc, 0u, partials, ticket, tot) && threadIdx.x == 0) st->est = sqrt(tot[0]);
}

__global__ void k_scale(long long n, double* __restrict__ v, const SolveState* st) {
    const double nv = st->est;
    const double inv = nv > 0 ? 1.0 / nv : 1.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) v[i] *= inv;
}

__global__ void k_lz_x(long long n, const double* __restrict__ invD, const double* __restrict__ v, double* __restrict__ x) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) x[i] = sqrt(invD[i]) * v[i];
}

// w = sq w - b vp (b = |w| of the previous step, 0 on the first); alpha = w . v into *aOut
__global__ void k_lz_w(long long n, const double* __restrict__ invD, double* __restrict__ w, const double* __restrict__ v,
                       const double* __restrict__ vp, const double* bPrev, double* aOut, SolveState* st, double* partials, unsigned* ticket) {
    const double b = bPrev ? *bPrev : 0.0;
    double acc[1] = {0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double wv = sqrt(invD[i]) * w[i] - b * vp[i];
        w[i] = wv;
        acc[0] += wv * v[i];
    }
    double tot[1];
    if (gridReduce<1>(acc, 0u, partials, ticket, tot) && threadIdx.x == 0) *aOut = tot[0];
}

// w -= alpha v; |w| into *bOut
__global__ void k_lz_axpy(long long n, double* __restrict__ w, const double* __restrict__ v, const double* aIn, double* bOut, SolveState* st,
                          double* partials, unsigned* ticket) {
    const double a = *aIn;
    double acc[1] = {0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double wv = w[i] - a * v[i];
        w[i] = wv;
        acc[0] += wv * wv;
    }
    double tot[1];
    if (gridReduce<1>(acc, 0u, partials, ticket, tot) && threadIdx.x == 0) *bOut = sqrt(tot[0]);
}

// vp = v; v = w / b (after the sequence has stopped these values are never used)
__global__ void k_lz_next(long long n, const double* __restrict__ w, double* __restrict__ v, double* __restrict__ vp, const double* bIn) {
    const double b = *bIn;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        vp[i] = v[i];
        v[i] = w[i] / b;
    }
}

// ---- the C ABI's dense layout (node i + NX (j + NY k)) <-> the pitched device layout (i + PX (j + NY k))

template <class T>
__global__ void k_pitch(const T* __restrict__ src, T* __restrict__ dst, int comps, int NX, int NY, int NZ, int PX, int toPitched) {
    const long long total = (long long)NX * NY * NZ * comps;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const long long nd = e / comps, row = nd / NX;
        const int c = int(e - nd * comps), i = int(nd - row * NX);
        const long long ep = (i + (long long)PX * row) * comps + c;
        if (toPitched) dst[ep] = src[e];
        else dst[e] = src[ep];
    }
}

// ---- post-processing: nodal stresses (voxel_fea.cpp:968-1037) and reactions (:929-940)

struct StressCoefs {
    double S[8][144];  // corner stress matrices times E / h, [a][row * 24 + q]
};

__device__ void principals3(double sx, double sy, double sz, double txy, double tyz, double tzx, double out[3]) {
    // eigenvalues of the symmetric stress tensor by the trigonometric solution of its cubic
    const double p1 = txy * txy + tyz * tyz + tzx * tzx;
    const double q = (sx + sy + sz) / 3;
    const double sc = fabs(sx) + fabs(sy) + fabs(sz) + sqrt(p1);
    if (p1 <= 1e-24 * sc * sc) {
        double a = sx, b = sy, c = sz, t;
        if (a < b) { t = a; a = b; b = t; }
        if (b < c) { t = b; b = c; c = t; }
        if (a < b) { t = a; a = b; b = t; }
        out[0] = a; out[1] = b; out[2] = c;
        return;
    }
    const double p2 = (sx - q) * (sx - q) + (sy - q) * (sy - q) + (sz - q) * (sz - q) + 2 * p1;
    const double p = sqrt(p2 / 6);
    const double b11 = (sx - q) / p, b22 = (sy - q) / p, b33 = (sz - q) / p, b12 = txy / p, b23 = tyz / p, b13 = tzx / p;
    const double det = b11 * (b22 * b33 - b23 * b23) - b12 * (b12 * b33 - b23 * b13) + b13 * (b12 * b23 - b22 * b13);
    const double rr = fmin(1.0, fmax(-1.0, det / 2));
    const double phi = acos(rr) / 3;
    out[0] = q + 2 * p * cos(phi);
    out[2] = q + 2 * p * cos(phi + 2.0943951023931954923);
    out[1] = 3 * q - out[0] - out[2];
}

__global__ void __launch_bounds__(NODE_THREADS) k_stresses(LevelView L, StressCoefs SC, const double* __restrict__ u, int principals,
                                                           float* __restrict__ vm, float* __restrict__ p1, float* __restrict__ p3) {
    const long long NX = L.PX, NXY = (long long)L.PX * L.NY;
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < L.nNodes; n += (long long)gridDim.x * blockDim.x) {
        const uint8_t mask = L.nmask[n];
        float ovm = 0, op1 = 0, op3 = 0;
        if (mask & NM_ACTIVE) {
            int i, j, k;
            nodeCoords(L, n, i, j, k);
            double svm = 0, sp1 = 0, sp3 = 0, wsum = 0;
#pragma unroll
            for (int v = 0; v < 8; v++) {
                const int di = v & 1, dj = (v >> 1) & 1, dk = v >> 2;
                const int ei = i - 1 + di, ej = j - 1 + dj, ek = k - 1 + dk;
                if (ei < 0 || ej < 0 || ek < 0 || ei >= L.nx || ej >= L.ny || ek >= L.nz) continue;
                const uint32_t w = L.word[L.wi(ei, ej, ek)];
                if (w == 0) continue;
                const int a = cornerOf(1 - di, 1 - dj, 1 - dk);
                double sig[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
                for (int b = 0; b < 8; b++) {
                    const int bx = (b == 1 || b == 2 || b == 5 || b == 6), by = (b == 2 || b == 3 || b == 6 || b == 7), bz = b >> 2;
                    const double* xp = u + 3 * (n + (di + bx - 1) + (dj + by - 1) * NX + (dk + bz - 1) * NXY);
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        const double xv = xp[c];
#pragma unroll
                        for (int rr = 0; rr < 6; rr++) sig[rr] += SC.S[a][rr * 24 + 3 * b + c] * xv;
                    }
                }
                const double rho = double(__uint_as_float(w));
                svm += rho * sqrt(0.5 * ((sig[0] - sig[1]) * (sig[0] - sig[1]) + (sig[1] - sig[2]) * (sig[1] - sig[2]) +
                                         (sig[2] - sig[0]) * (sig[2] - sig[0])) +
                                  3 * (sig[3] * sig[3] + sig[4] * sig[4] + sig[5] * sig[5]));
                if (principals) {
                    double pr[3];
                    principals3(sig[0], sig[1], sig[2], sig[3], sig[4], sig[5], pr);
                    sp1 += rho * pr[0];
                    sp3 += rho * pr[2];
                }
                wsum += rho;
            }
            if (wsum > 0) {
                ovm = float(svm / wsum);
                op1 = float(sp1 / wsum);
                op3 = float(sp3 / wsum);
            }
        }
        vm[n] = ovm;
        if (principals) {
            p1[n] = op1;
            p3[n] = op3;
        }
    }
}

__global__ void k_reactions(long long nNodes, const uint8_t* __restrict__ nmask, const uint8_t* __restrict__ bc, const double* __restrict__ y,
                            const double* __restrict__ f, SolveState* st, double* partials, unsigned* ticket) {
    double v[3] = {0, 0, 0};
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < nNodes; n += (long long)gridDim.x * blockDim.x) {
        if (!(nmask[n] & NM_ACTIVE)) continue;
#pragma unroll
        for (int c = 0; c < 3; c++)
            if (bc[3 * n + c]) v[c] += y[3 * n + c] - (f ? f[3 * n + c] : 0.0);
    }
    double tot[3];
    if (gridReduce<3>(v, 0u, partials, ticket, tot) && threadIdx.x == 0) {
        st->alpha = tot[0];
        st->beta = tot[1];
        st->pq = tot[2];
    }
}

}  // namespace dev
}  // namespace psfea

#include "block_kernels.cuh"  // the multi-RHS kernels (they use the control helpers above)
#include "ebe_kernels.cuh"    // the tensor-core element-block operator
#include "block_tc.cuh"       // the block operator on the tensor cores
#include "stencil_kernels.cuh"  // assembled stencils of the Galerkin levels

namespace psfea {
namespace dev {

// A list-driven FP32 pass (APPLY / CHEB / RESID) over a level's nodes: the boundary nodes of a split
// level, or every active node of a sparse level (a thin-walled lattice leaves two thirds of a
// tile's node slots inactive, and the tiles still stage and store them). Each node's 27 neighbours
// are read once, two z-planes at a time (81 loads instead of up to 192 in the per-voxel gather).
// CLS: the level's Galerkin matrices come in few classes; each CTA (persistent, one per SM) first
// copies them all into shared memory and gathers the rows from there. The sums are those of k_bnd
// in the same order (bitwise the same results); nodes off the list are not written.
// V = __half: the FP16 coarse-level vectors, iterates (x, d, y of CHEB) stored as x * sx and
// residuals (r, y of RESID) as r * sr with powers of two sx, sr; rho = sr / sx brings K x to the
// residual's scale and the caller passes c2 / rho (exact: powers of two). V = float: rho = 1.
template <int MODE, bool OWN16, bool CLS, class V = float>
__global__ void __launch_bounds__(512) k_list(LevelView L, Coefs<float> C, const int* __restrict__ list, int count, int nClass,
                                               const V* __restrict__ x, V* __restrict__ y, const V* __restrict__ r, V* __restrict__ d,
                                               float c1, float c2, float rho, int raw, Ctl ctl) {
    if (skipped(ctl)) return;
    extern __shared__ __align__(16) unsigned char clsRaw[];
    LevelView Ls = L;
    if constexpr (CLS) {
        const size_t bytes = size_t(nClass) * 576 * (OWN16 ? 2 : 4);
        const uint4* src = reinterpret_cast<const uint4*>(OWN16 ? static_cast<const void*>(L.own16) : static_cast<const void*>(L.own));
        uint4* dst = reinterpret_cast<uint4*>(clsRaw);
        for (size_t e = threadIdx.x; e < bytes / 16; e += blockDim.x) dst[e] = __ldg(src + e);
        __syncthreads();
        if (OWN16) Ls.own16 = reinterpret_cast<const __half*>(clsRaw);
        else Ls.own = reinterpret_cast<const float*>(clsRaw);
    }
    constexpr bool H = !std::is_same<V, float>::value;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < count; t += (long long)gridDim.x * blockDim.x) {
        const long long n = list[t];
        const uint8_t mask = __ldg(L.nmask + n);
        int i, j, k;
        nodeCoords(L, n, i, j, k);
        float acc[3];
        applyNbr<float, OWN16, 1, CLS, V>(Ls, C, x, i, j, k, n, mask, acc);
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const long long id = 3 * n + q;
            const bool fx = fixedDof(mask, q);
            const float kx = H ? rho * acc[q] : acc[q];
            if (MODE == TOP_APPLY) {
                stv(y + id, (!raw && fx) ? 0.f : kx);
            } else if (MODE == TOP_RESID) {
                stv(y + id, fx ? 0.f : ldf(r + id) - kx);
            } else {
                if (fx) {
                    stv(d + id, 0.f);
                    stv(y + id, 0.f);
                } else {
                    const float dn = c1 * ldf(d + id) + c2 * L.invD[id] * (ldf(r + id) - kx);
                    stv(d + id, dn);
                    stv(y + id, ldf(x + id) + dn);
                }
            }
        }
    }
}

}  // namespace dev
}  // namespace psfea

namespace psfea {

// ==================================================================== host side

namespace {

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        if (e == cudaErrorMemoryAllocation) throw Error(PS_EOOM, std::string(what) + ": " + cudaGetErrorString(e));
        if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) throw Error(PS_ENODEV, std::string(what) + ": " + cudaGetErrorString(e));
        throw Error(PS_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

// Device buffer. With a stream it is allocated and freed stream-ordered (cudaMallocAsync /
// cudaFreeAsync), which never waits for the rest of the device: handles come and go while other
// solves run (serving). Without one it uses cudaMalloc / cudaFree.
struct DevMem {
    void* p = nullptr;
    size_t bytes = 0;
    cudaStream_t s = nullptr;
    DevMem() = default;
    DevMem(const DevMem&) = delete;
    DevMem& operator=(const DevMem&) = delete;
    DevMem(DevMem&& o) noexcept : p(o.p), bytes(o.bytes), s(o.s) { o.p = nullptr; o.bytes = 0; }
    DevMem& operator=(DevMem&&) = delete;  // buffers move only into new owners (vector growth)
    ~DevMem() { release(); }
    void release() {
        if (p) {
            if (s) cudaFreeAsync(p, s);
            else cudaFree(p);
        }
        p = nullptr;
        bytes = 0;
    }
    void alloc(size_t n, int64_t& total, cudaStream_t stream = nullptr) {
        release();
        s = stream;
        if (n == 0) return;
        if (s) {
            check(cudaMallocAsync(&p, n, s), "cudaMallocAsync");
            check(cudaMemsetAsync(p, 0, n, s), "cudaMemsetAsync");
        } else {
            check(cudaMalloc(&p, n), "cudaMalloc");
            check(cudaMemset(p, 0, n), "cudaMemset");
        }
        bytes = n;
        total += int64_t(n);
    }
    template <class T> T* as() const { return static_cast<T*>(p); }
};

// a level's per-node (comps 1) or per-DOF (comps 3) host array in the pitched device layout,
// padding entries `fill`
// (rows copied over the host threads, converted to T on the way, padding written per row)
template <class T, class S, class A>
std::vector<T, UninitAlloc<T>> pitched(const std::vector<S, A>& v, int comps, const HostLevel& h, int PX, T fill) {
    std::vector<T, UninitAlloc<T>> o(size_t(PX) * h.NY * h.NZ * comps);
    const size_t rowIn = size_t(h.NX) * comps, rowOut = size_t(PX) * comps;
    parallelFor(int64_t(h.NY) * h.NZ, [&](int64_t r0, int64_t r1) {
        for (int64_t row = r0; row < r1; row++) {
            T* out = o.data() + row * rowOut;
            const S* in = v.data() + row * rowIn;
            for (size_t q = 0; q < rowIn; q++) out[q] = T(in[q]);
            for (size_t q = rowIn; q < rowOut; q++) out[q] = fill;
        }
    }, 1024);
    return o;
}
std::vector<uint32_t> pitchedWords(const HostLevel& h, int px) {
    std::vector<uint32_t> o(size_t(px) * h.ny * h.nz, 0u);
    for (int64_t row = 0; row < int64_t(h.ny) * h.nz; row++)
        std::copy(h.word.begin() + row * h.nx, h.word.begin() + (row + 1) * h.nx, o.begin() + row * px);
    return o;
}
inline int pitch4(int n) { return (n + 3) & ~3; }

template <class T, class A>
void upload(DevMem& m, const std::vector<T, A>& v, int64_t& total, cudaStream_t s = nullptr) {
    m.alloc(v.size() * sizeof(T), total, s);
    if (!v.empty()) {
        if (s) check(cudaMemcpyAsync(m.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s), "upload");
        else check(cudaMemcpy(m.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
    }
}

int gridFor(int64_t n, int threads, int cap) {
    const int64_t b = (n + threads - 1) / threads;
    return int(std::max<int64_t>(1, std::min<int64_t>(b, cap)));
}

}  // namespace

// ---- tensor maps of the tiled kernels (cuTensorMapEncodeTiled through the runtime's driver entry
// point, so the library needs no link to the driver library)
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encodeTiled() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
        else
            cudaGetLastError();
    });
    if (!fn) throw Error(PS_ECUDA, "cuTensorMapEncodeTiled is not available from the driver");
    return fn;
}

enum MapKind { MAP_HALO = 0, MAP_TILE = 1, MAP_WORDS = 2 };

// x halo boxes (PROW x HY x HZ values), tile boxes (TROW x TY x TZ) over a level's pitched DOF
// vector, or voxel-word boxes (WROW x VY x VZ); outside the tensor loads read 0 and stores are dropped
CUtensorMap makeMap(const void* base, MapKind kind, bool f64, const dev::LevelView& v) {
    CUtensorMap m;
    cuuint64_t dims[3];
    cuuint32_t box[3];
    const cuuint32_t es[3] = {1, 1, 1};
    CUtensorMapDataType dt;
    size_t esz;
    if (kind == MAP_WORDS) {
        dt = CU_TENSOR_MAP_DATA_TYPE_UINT32;
        esz = 4;
        dims[0] = cuuint64_t(v.px); dims[1] = cuuint64_t(v.ny); dims[2] = cuuint64_t(v.nz);
        box[0] = dev::WROW; box[1] = dev::VY; box[2] = dev::VZ;
    } else {
        dt = f64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
        esz = f64 ? 8 : 4;
        dims[0] = cuuint64_t(3) * v.PX; dims[1] = cuuint64_t(v.NY); dims[2] = cuuint64_t(v.NZ);
        if (kind == MAP_HALO) { box[0] = dev::PROW; box[1] = dev::HY; box[2] = dev::HZ; }
        else { box[0] = dev::TROW; box[1] = dev::TY; box[2] = dev::TZ; }
    }
    const cuuint64_t strides[2] = {dims[0] * esz, dims[0] * dims[1] * esz};
    const CUresult r = encodeTiled()(&m, dt, 3, const_cast<void*>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                     CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Error(PS_ECUDA, "cuTensorMapEncodeTiled failed (" + std::to_string(int(r)) + ")");
    return m;
}

// Read-only device data of one level, shared by every solve context of a handle.
struct DevLevel {
    dev::LevelView view{};
    dev::Coefs<double> c64{};
    dev::Coefs32 c32{};
    DevMem word, nmask, own, own16, invD, dadd, dadd32, bc;
    DevMem tiles;      // packed (tx, ty, tz) of the 32 x 8 x 4 node tiles with an active node
    int nTiles = 0;
    DevMem blist;      // tiled levels: the boundary nodes (pitched indices, increasing)
    int nBnd = 0;
    bool inner64 = false;  // 64-bit tiles compute their boundary nodes themselves (else k_bnd does)
    bool split32 = false;  // 32-bit tiles leave their boundary nodes to k_bnd (else they compute them)
    bool useTiles = false;  // tiled kernel (large levels) or one thread per node (small ones)
    bool use8 = false;      // eight lanes per node (the smallest levels)
    float cf0 = 0, cf1 = 0, cf2 = 0, omega = 0.5f;
    std::vector<float> chebC1, chebC2;  // steps 1 .. degree-1 of the Chebyshev smoother: d = c1 d + c2 D^-1 (r - K z)
    bool hasOwn = false;
    int nOwnDev = 0;  // own matrices on the device (classes when they are shared)
    // the tensor-core element-block operator (levels without Galerkin matrices): its 8 x 8 x 4 tiles
    DevMem ebeTiles;
    int nEbeTiles = 0;
    bool ebe = false;
    // assembled stencils (levels >= 1): of the boundary nodes of a split tiled level, or of every
    // active node of an untiled one (stnNodes: those nodes, in order); FP32 and the FP16 copy
    // over the power-of-two scale stnScale, each made on first use
    const int* stnNodes = nullptr;
    int nStn = 0;
    DevMem stn32, stn16;
    float stnScale = 1.f;
    void release() {
        for (DevMem* b : {&word, &nmask, &own, &own16, &invD, &dadd, &dadd32, &bc, &tiles, &blist, &ebeTiles, &stn32, &stn16}) b->release();
    }
};

// The V-cycle work vectors of one level in one solve context.
struct LevelWork {
    DevMem r, z, t, d;
    void release() {
        for (DevMem* b : {&r, &z, &t, &d}) b->release();
    }
};

// The hierarchy on the device: built once per handle, shared by its solve contexts.
struct SharedModel {
    Hierarchy H;
    std::vector<DevLevel> L;
    DevMem cDof, cInv;  // coarsest level: free DOF list, dense FP64 inverse
    int m = 0;
    int64_t bytes = 0;
    int smCount = 148;
    int devId = 0;  // the CUDA device the model's data lives on
    int maxTiles = 0;
    // smoother coefficients (shared; `version` changes whenever they do, so contexts re-record)
    bool smoothersReady = false;
    int degree = 2;  // Chebyshev smoother degree (the reference's is 2)
    int defaultDegree = 2;  // the degree of solves that leave it open (an autotuned model's choice)
    int64_t version = 0;
    // FP16 own matrices (mixed precision) may be applied to neighbour differences, keeping rigid
    // translations in their null space exactly despite the rounding of the entries; the mixed form
    // may also keep the 32-bit matrices. Tuning knobs: PSFEA_OWN16_DIFF, PSFEA_MIXED_OWN32, PSFEA_FOLD.
    bool ownDiff = false;
    bool mixedOwn16 = true;
    bool ownDedup = true;  // one device copy per class of equal own matrices (PSFEA_OWN_DEDUP=0: one per voxel)
    double foldFactor = 0.1;  // fold when the FP32 residual is this fraction of its peak
    // reduced-precision forms: levels (bit l) whose FP32 operator runs on the tensor cores
    // (element-block form, levels without Galerkin matrices only), and its TF32 split (1 or 3 terms).
    // PSFEA_EBE, PSFEA_EBE_SPLIT
    int64_t ebeLevels = 0;
    int ebeSplit = 3;
    // boundary passes gather Galerkin classes from shared memory when they fit in this many bytes
    // (PSFEA_CLS_SMEM; 0 = never)
    size_t clsSmemMax = 200 * 1024;
    // levels (bit l) whose FP32 passes run over their active-node list instead of tiles or one
    // thread per pitched node (PSFEA_LIST_LEVELS)
    int64_t listLevels = 0;
    // PS_PREC_HALF: per level the power of two delta_l (iterates stored as x * 8^-l * delta_l,
    // residuals as r * 8^-l) and the inner solve's refinement factor
    std::vector<float> halfDelta;
    bool halfOk = false;  // every level >= 1 fits FP16 with its scale
    double refineEta = 0.1;
    std::mutex listMu;
    std::atomic<bool> actReady{false};  // act / nAct complete for every level
    cudaStream_t ms = nullptr;     // allocation / upload stream of the shared data
    cudaEvent_t readyEv = nullptr; // recorded when the uploads are done; contexts wait on it

    ~SharedModel() {
        for (auto& a : act) a.release();
        for (auto& b : bstn32) b.release();
        btTiles.release();
        for (auto& D : L) D.release();
        cDof.release();
        cInv.release();
        if (ms) {
            cudaStreamSynchronize(ms);
            cudaStreamDestroy(ms);
        }
        if (readyEv) cudaEventDestroy(readyEv);
    }

    // per level, the pitched indices of its active nodes in increasing order (the block kernels walk
    // them); built on the first block solve
    std::vector<DevMem> act;
    std::vector<int> nAct;
    // the finest level's 8 x 4 x 4 node tiles with an active node, for the block tensor-core
    // operator (built with the active lists); PSFEA_BLOCK_TC=1 runs the mixed block form's finest
    // level on it (measured slower than the CUDA-core block kernel, so off by default)
    DevMem btTiles;
    int nBtTiles = 0;
    bool blockTc = false;

    void build(const int32_t dims[3], const float* density, double nu, const uint8_t* bc, int64_t coarsest, const double* diagAdd);
    void adopt(Hierarchy&& h);  // upload a hierarchy built on the host beforehand
    void uploadLevel(int l);
    void ensureActiveLists();
    // the assembled stencils of the levels in stencilLevels (FP16 copies too when half); the
    // callers' streams wait on readyEv
    void ensureStencils(bool half);
    // the block path's stencils: FP32 over the active nodes of every level below the finest
    // (PSFEA_BLOCK_STENCIL=0: none, the per-voxel gather)
    void ensureBlockStencils();
    std::vector<DevMem> bstn32;
    bool blockStencils = true;
    // PSFEA_BLOCK_STENCIL0=1: stencils on the finest level too. Off: its uniform element matrix is a
    // kernel operand, and measured on the SIMP block solve its stencils were 16-20 % slower (paired
    // or not) than the constant-operand gather
    bool blockStencil0 = false;
    int64_t stencilLevels = ~int64_t(1);  // PSFEA_STENCIL_LEVELS: bit l = level l (never level 0)
    int64_t stencilMinNodes = 65536;      // PSFEA_STENCIL_MIN_NODES: smaller node lists keep the gather
    bool foldBranch = true;               // PSFEA_FOLD_BRANCH: the FP32-Krylov fold as a conditional graph branch
    bool exactOneLevel() const { return L.size() == 1 && H.hasFactor(); }
};

void SharedModel::build(const int32_t dims[3], const float* density, double nu, const uint8_t* bc, int64_t coarsest, const double* diagAdd) {
    // PSFEA_DEVICE_GALERKIN=1: the own matrices of graded coarse levels are computed on this device
    // (bitwise the host's). Off by default: measured on a 16-core host, the SIMP grid 192x96x96
    // builds in 0.12 s on the host threads against 0.30 s with the device products, whose 415 MB of
    // level-1 matrices come back over PCIe for the host's diagonal, class and upload steps.
    std::unique_ptr<GalerkinEngine> engine;
    const char* e = std::getenv("PSFEA_DEVICE_GALERKIN");
    if (e && std::atoi(e) != 0) engine = makeDeviceGalerkin();
    adopt(buildHierarchy(dims, density, nu, bc, coarsest, diagAdd, engine.get()));
}

void SharedModel::adopt(Hierarchy&& h) {
    H = std::move(h);
    check(cudaGetDevice(&devId), "cudaGetDevice");
    check(cudaDeviceGetAttribute(&smCount, cudaDevAttrMultiProcessorCount, devId), "attribute");
    if (const char* e = std::getenv("PSFEA_OWN16_DIFF")) ownDiff = std::atoi(e) != 0;
    if (const char* e = std::getenv("PSFEA_FOLD")) foldFactor = std::atof(e);
    if (const char* e = std::getenv("PSFEA_MIXED_OWN32")) mixedOwn16 = std::atoi(e) == 0;
    if (const char* e = std::getenv("PSFEA_OWN_DEDUP")) ownDedup = std::atoi(e) != 0;
    if (const char* e = std::getenv("PSFEA_EBE")) ebeLevels = std::atoll(e);
    if (const char* e = std::getenv("PSFEA_CLS_SMEM")) clsSmemMax = size_t(std::atoll(e));
    if (const char* e = std::getenv("PSFEA_LIST_LEVELS")) listLevels = std::atoll(e);
    if (const char* e = std::getenv("PSFEA_REFINE_ETA")) refineEta = std::atof(e);
    if (const char* e = std::getenv("PSFEA_STENCIL_LEVELS")) stencilLevels = std::atoll(e) & ~int64_t(1);
    if (const char* e = std::getenv("PSFEA_STENCIL_MIN_NODES")) stencilMinNodes = std::atoll(e);
    if (const char* e = std::getenv("PSFEA_FOLD_BRANCH")) foldBranch = std::atoi(e) != 0;
    if (const char* e = std::getenv("PSFEA_BLOCK_STENCIL")) blockStencils = std::atoi(e) != 0;
    if (const char* e = std::getenv("PSFEA_BLOCK_STENCIL0")) blockStencil0 = std::atoi(e) != 0;
    if (const char* e = std::getenv("PSFEA_EBE_SPLIT")) ebeSplit = std::atoi(e) == 1 ? 1 : 3;
    check(cudaStreamCreateWithFlags(&ms, cudaStreamNonBlocking), "stream");
    check(cudaEventCreateWithFlags(&readyEv, cudaEventDisableTiming), "event");
    static std::once_flag attrOnce;
    std::call_once(attrOnce, [] {
        // the tiled operator stages more than the default 48 KB of shared memory
        auto set = [](auto kernel, size_t bytes) {
            check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)), "attr");
        };
        set(dev::k_tile<double, dev::TOP_APPLY, false, false>, dev::tileSmemBytes<double, dev::TOP_APPLY, false>());
        set(dev::k_tile<double, dev::TOP_DOT, false, false>, dev::tileSmemBytes<double, dev::TOP_DOT, false>());
        set(dev::k_tile<double, dev::TOP_APPLY, false, false, true>, dev::tileSmemBytes<double, dev::TOP_APPLY, true>());
        set(dev::k_tile<double, dev::TOP_DOT, false, false, true>, dev::tileSmemBytes<double, dev::TOP_DOT, true>());
        set(dev::k_tile<float, dev::TOP_CHEB, false, false>, dev::tileSmemBytes<float, dev::TOP_CHEB, true>());
        set(dev::k_tile<float, dev::TOP_CHEB, true, false>, dev::tileSmemBytes<float, dev::TOP_CHEB, true>());
        set(dev::k_tile<float, dev::TOP_CHEB, true, true>, dev::tileSmemBytes<float, dev::TOP_CHEB, true>());
        set(dev::k_tile<float, dev::TOP_RESID, false, false>, dev::tileSmemBytes<float, dev::TOP_RESID, true>());
        set(dev::k_tile<float, dev::TOP_RESID, true, false>, dev::tileSmemBytes<float, dev::TOP_RESID, true>());
        set(dev::k_tile<float, dev::TOP_RESID, true, true>, dev::tileSmemBytes<float, dev::TOP_RESID, true>());
        set(dev::k_tile<float, dev::TOP_DOT, false, true>, dev::tileSmemBytes<float, dev::TOP_DOT, true>());
        set(dev::k_tile<float, dev::TOP_CHEB, false, false, false>, dev::tileSmemBytes<float, dev::TOP_CHEB, false>());
        set(dev::k_tile<float, dev::TOP_CHEB, true, false, false>, dev::tileSmemBytes<float, dev::TOP_CHEB, false>());
        set(dev::k_tile<float, dev::TOP_CHEB, true, true, false>, dev::tileSmemBytes<float, dev::TOP_CHEB, false>());
        set(dev::k_tile<float, dev::TOP_RESID, false, false, false>, dev::tileSmemBytes<float, dev::TOP_RESID, false>());
        set(dev::k_tile<float, dev::TOP_RESID, true, false, false>, dev::tileSmemBytes<float, dev::TOP_RESID, false>());
        set(dev::k_tile<float, dev::TOP_RESID, true, true, false>, dev::tileSmemBytes<float, dev::TOP_RESID, false>());
        set(dev::k_ebe<dev::TOP_APPLY, 1>, dev::ebeSmemBytes<1>());
        set(dev::k_ebe<dev::TOP_CHEB, 1>, dev::ebeSmemBytes<1>());
        set(dev::k_ebe<dev::TOP_RESID, 1>, dev::ebeSmemBytes<1>());
        set(dev::k_ebe<dev::TOP_APPLY, 3>, dev::ebeSmemBytes<3>());
        set(dev::k_ebe<dev::TOP_CHEB, 3>, dev::ebeSmemBytes<3>());
        set(dev::k_ebe<dev::TOP_RESID, 3>, dev::ebeSmemBytes<3>());
        set(dev::k_list<dev::TOP_CHEB, true, true>, 200 * 1024);
        set(dev::k_list<dev::TOP_CHEB, false, true>, 200 * 1024);
        set(dev::k_list<dev::TOP_RESID, true, true>, 200 * 1024);
        set(dev::k_list<dev::TOP_RESID, false, true>, 200 * 1024);
        set(dev::k_list<dev::TOP_APPLY, true, true>, 200 * 1024);
        set(dev::k_list<dev::TOP_APPLY, false, true>, 200 * 1024);
        set(dev::k_list<dev::TOP_CHEB, true, true, __half>, 200 * 1024);
        set(dev::k_list<dev::TOP_CHEB, false, true, __half>, 200 * 1024);
        set(dev::k_list<dev::TOP_RESID, true, true, __half>, 200 * 1024);
        set(dev::k_list<dev::TOP_RESID, false, true, __half>, 200 * 1024);
        set(dev::kb_tc<dev::BOP_APPLY>, dev::btSmemBytes());
        set(dev::kb_tc<dev::BOP_CHEB>, dev::btSmemBytes());
        set(dev::kb_tc<dev::BOP_RESID>, dev::btSmemBytes());
    });
    L.resize(H.levels.size());
    for (int l = 0; l < int(H.levels.size()); l++) uploadLevel(l);
    m = int(H.coarseM);
    if (H.hasFactor()) {
        // the coarsest level's free DOFs as pitched indices
        const HostLevel& hc = H.levels.back();
        const int PX = L.back().view.PX;
        std::vector<int32_t> dofs(H.coarseDof.size());
        for (size_t q = 0; q < dofs.size(); q++) {
            const int64_t e = H.coarseDof[q], nd = e / 3, row = nd / hc.NX;
            dofs[q] = int32_t(3 * ((nd - row * hc.NX) + int64_t(PX) * row) + (e - 3 * nd));
        }
        upload(cDof, dofs, bytes, ms);
        upload(cInv, H.coarseInv, bytes, ms);
    }
    for (auto& D : L) maxTiles = std::max(maxTiles, D.nTiles);
    // delta_l = 2^(round(log2(median diagonal of level l)) - 4): the FP16 iterates then sit near
    // 1/16 of the residuals' order one, leaving room for the coarse corrections' growth
    // (one scale per level cannot hold graded stiffness in FP16: when a level's diagonal spans more
    // than 2^8, e.g. SIMP densities down to 1e-3 with p = 3, the form keeps FP32 coarse vectors)
    halfDelta.assign(L.size(), 1.f);
    halfOk = L.size() > 1;
    for (size_t l = 1; l < L.size(); l++) {
        const auto& inv = H.levels[l].invDiag;
        double lo = 0, hi = 0;
        std::vector<double> dg;
        const size_t stride = std::max<size_t>(1, inv.size() / 65536);
        for (size_t q = 0; q < inv.size(); q++)
            if (inv[q] > 0) {
                const double v = 1.0 / inv[q];
                lo = lo > 0 ? std::min(lo, v) : v;
                hi = std::max(hi, v);
                if (q % stride == 0) dg.push_back(v);
            }
        if (dg.empty()) continue;
        if (hi > 256.0 * lo) halfOk = false;
        std::nth_element(dg.begin(), dg.begin() + dg.size() / 2, dg.end());
        const int e = int(std::lround(std::log2(dg[dg.size() / 2]))) - 4;
        halfDelta[l] = std::ldexp(1.f, std::max(-120, std::min(120, e)));
    }
    if (listLevels) ensureActiveLists();
    check(cudaEventRecord(readyEv, ms), "event");
}

void SharedModel::uploadLevel(int l) {
    const HostLevel& h = H.levels[size_t(l)];
    DevLevel& D = L[size_t(l)];
    const int PX = pitch4(h.NX), px = pitch4(h.nx);
    std::vector<uint32_t> words = pitchedWords(h, px);
    // ownDedup: one device copy per class of bitwise-equal own matrices (the hierarchy's classes),
    // the voxel words pointing at it. Every kernel reads a matrix through its voxel's word, so the
    // results do not change; lattices and solid/void parts have tens to hundreds of classes for
    // 10^4-10^6 matrices (graded grids have none to share and keep their arrays).
    const std::vector<float, UninitAlloc<float>>* ownSrc = &h.own;
    std::vector<float, UninitAlloc<float>> classes;
    if (ownDedup && h.nOwn > 0 && int64_t(h.ownClass.size()) == h.nOwn) {
        int32_t nClass = 0;
        for (int32_t c : h.ownClass) nClass = std::max(nClass, c + 1);
        if (nClass < h.nOwn) {
            classes.resize(size_t(nClass) * 576);
            std::vector<uint8_t> seen(size_t(nClass), 0);
            for (int64_t o = 0; o < h.nOwn; o++) {
                const int32_t c = h.ownClass[size_t(o)];
                if (seen[size_t(c)]) continue;
                seen[size_t(c)] = 1;
                std::memcpy(classes.data() + size_t(c) * 576, h.own.data() + size_t(o) * 576, 576 * sizeof(float));
            }
            for (uint32_t& w : words)
                if (w & OWN_BIT) w = OWN_BIT | uint32_t(h.ownClass[w & ~OWN_BIT]);
            ownSrc = &classes;
        }
    }
    const auto& own = *ownSrc;
    D.nOwnDev = int(own.size() / 576);
    upload(D.word, words, bytes, ms);
    upload(D.nmask, pitched<uint8_t>(h.nmask, 1, h, PX, uint8_t(7)), bytes, ms);  // padding: inactive, all held
    D.hasOwn = h.nOwn > 0;
    if (D.hasOwn) {
        upload(D.own, own, bytes, ms);
        // halves with a power-of-two level scale keeping the largest entry near 2^14
        // (the largest entry by chunks over the host threads: the max does not depend on the split)
        const int64_t nEnt = int64_t(own.size()), chunk = int64_t(1) << 20;
        std::vector<double> cmax(size_t((nEnt + chunk - 1) / chunk), 0.0);
        parallelFor(int64_t(cmax.size()), [&](int64_t c0, int64_t c1) {
            for (int64_t c = c0; c < c1; c++) {
                float m = 0.f;
                for (int64_t i = c * chunk, e = std::min(nEnt, (c + 1) * chunk); i < e; i++) m = std::max(m, std::fabs(own[size_t(i)]));
                cmax[size_t(c)] = double(m);
            }
        }, 1);
        double kmax = 0;
        for (double v : cmax) kmax = std::max(kmax, v);
        const float hs = kmax > 0 ? float(std::exp2(std::ceil(std::log2(kmax / 16384.0)))) : 1.f;
        std::vector<__half, UninitAlloc<__half>> h16(own.size());  // every entry written below
        const float inv = 1.f / hs;
        parallelFor(int64_t(own.size()), [&](int64_t lo, int64_t hi) {
            for (int64_t i = lo; i < hi; i++) h16[size_t(i)] = __float2half_rn(own[size_t(i)] * inv);
        });
        upload(D.own16, h16, bytes, ms);
        D.view.hs = hs;
    }
    upload(D.invD, pitched<float>(h.invDiag, 3, h, PX, 0.f), bytes, ms);
    if (!h.diagAdd.empty()) {
        upload(D.dadd, pitched<double>(h.diagAdd, 3, h, PX, 0.0), bytes, ms);
        upload(D.dadd32, pitched<float>(h.diagAdd, 3, h, PX, 0.f), bytes, ms);
    }
    if (l == 0) upload(D.bc, pitched<uint8_t>(h.bc, 3, h, PX, uint8_t(0)), bytes, ms);
    {
        const int ntx = (h.NX + dev::TX - 1) / dev::TX, nty = (h.NY + dev::TY - 1) / dev::TY, ntz = (h.NZ + dev::TZ - 1) / dev::TZ;
        if (ntx > 2047 || nty > 2047 || ntz > 1023) throw Error(PS_EINVAL, "grid too large for the tile index");
        std::vector<uint8_t> act(size_t(ntx) * nty * ntz, 0);
        for (int k = 0; k < h.NZ; k++)
            for (int j = 0; j < h.NY; j++) {
                const uint8_t* row = h.nmask.data() + h.node(0, j, k);
                for (int i = 0; i < h.NX; i++)
                    if (row[i] & NM_ACTIVE) act[size_t((i / dev::TX) + ntx * ((j / dev::TY) + size_t(nty) * (k / dev::TZ)))] = 1;
            }
        std::vector<uint32_t> list;
        for (int tz = 0; tz < ntz; tz++)
            for (int ty = 0; ty < nty; ty++)
                for (int tx = 0; tx < ntx; tx++)
                    if (act[size_t(tx + ntx * (ty + size_t(nty) * tz))]) list.push_back(dev::packTile(tx, ty, tz));
        D.nTiles = int(list.size());
        upload(D.tiles, list, bytes, ms);
        if (h.nOwn == 0 && l < 63 && ((ebeLevels >> l) & 1)) {
            // the element-block tiles (8 x 8 x 4 nodes) with an active node
            const int ex = (h.NX + dev::EX - 1) / dev::EX, ey = (h.NY + dev::EY - 1) / dev::EY, ez = (h.NZ + dev::EZ - 1) / dev::EZ;
            std::vector<uint8_t> ea(size_t(ex) * ey * ez, 0);
            for (int k = 0; k < h.NZ; k++)
                for (int j = 0; j < h.NY; j++) {
                    const uint8_t* row = h.nmask.data() + h.node(0, j, k);
                    for (int i = 0; i < h.NX; i++)
                        if (row[i] & NM_ACTIVE) ea[size_t((i / dev::EX) + ex * ((j / dev::EY) + size_t(ey) * (k / dev::EZ)))] = 1;
                }
            std::vector<uint32_t> el;
            for (int tz = 0; tz < ez; tz++)
                for (int ty = 0; ty < ey; ty++)
                    for (int tx = 0; tx < ex; tx++)
                        if (ea[size_t(tx + ex * (ty + size_t(ey) * tz))]) el.push_back(dev::packTile(tx, ty, tz));
            D.nEbeTiles = int(el.size());
            upload(D.ebeTiles, el, bytes, ms);
            D.ebe = D.nEbeTiles > 0;
        }
        // small levels have too few tiles to fill the GPU: one thread per node instead, or eight
        // lanes per node on the smallest ones
        int64_t minNodes = 400000;
        if (const char* e = std::getenv("PSFEA_TILE_MIN_NODES")) minNodes = std::atoll(e);
        // (and grids no smaller than the staging boxes of 116 x 10 x 6 values and 36 x 9 x 5 words)
        D.useTiles = h.nNodes >= minNodes && h.NY >= dev::HY && h.NZ >= dev::HZ && 3 * PX >= dev::PROW && px >= dev::WROW;
        int64_t max8 = 30000;
        if (const char* e = std::getenv("PSFEA_OP8_MAX_NODES")) max8 = std::atoll(e);
        D.use8 = !D.useTiles && l > 0 && h.nNodes <= max8;
        if (D.useTiles) {  // for the 64-bit tiled kernels
            std::vector<int32_t> bl(h.boundary.size());
            for (size_t q = 0; q < bl.size(); q++) {
                const int64_t nd = h.boundary[q], row = nd / h.NX;
                bl[q] = int32_t((nd - row * h.NX) + int64_t(PX) * row);
            }
            D.nBnd = int(bl.size());
            upload(D.blist, bl, bytes, ms);
            // in the tile once boundary nodes are a large share of the level (graded grids, thin
            // walls); PSFEA_TILE_INNER64: 0 never, 1 always
            int64_t active = 0;
            for (uint8_t mk : h.nmask) active += (mk & NM_ACTIVE) ? 1 : 0;
            D.inner64 = active > 0 && double(bl.size()) >= 0.3 * double(active);
            if (const char* e = std::getenv("PSFEA_TILE_INNER64")) {
                const int v = std::atoi(e);
                if (v == 0 || v == 1) D.inner64 = v == 1;
            }
            // 32-bit tiles of the Galerkin levels (l >= 1) leave their boundary nodes to k_bnd: there
            // the boundary nodes gather own matrices, and the few hundred tiles of such a level wait
            // on their heaviest ones (L-bracket level 1: 495 tiles, 36 % boundary nodes; FP64-form
            // solves 7-10 % faster on the L-bracket and the gyroid, the finest level slower split).
            // PSFEA_TILE_SPLIT32: bit l set = level l split
            D.split32 = l > 0;
            if (const char* e = std::getenv("PSFEA_TILE_SPLIT32")) D.split32 = l < 63 && ((std::atoll(e) >> l) & 1);
        }
    }
    dev::LevelView& v = D.view;
    v.nx = h.nx; v.ny = h.ny; v.nz = h.nz; v.NX = h.NX; v.NY = h.NY; v.NZ = h.NZ;
    v.PX = PX;
    v.px = px;
    v.nNodes = int64_t(PX) * h.NY * h.NZ;
    v.word = D.word.as<uint32_t>();
    v.nmask = D.nmask.as<uint8_t>();
    v.own = D.own.as<float>();
    v.own16 = D.own16.as<__half>();
    v.dadd = D.dadd.as<double>();
    v.dadd32 = D.dadd32.as<float>();
    v.invD = D.invD.as<float>();
    for (int i = 0; i < 576; i++) {
        D.c64.Kb[i] = h.Kb[i];
        D.c32.Kb[i] = float(h.Kb[i]);
    }
    for (int m = 0; m < 27; m++)
        for (int e = 0; e < 9; e++) {
            D.c64.S[m * 9 + e] = h.S[m][e];
            D.c32.S[m * 9 + e] = float(h.S[m][e]);
            D.c32.S2[m * 9 + e] = make_float2(float(h.S[m][e]), float(h.S[m][e]));
        }
}

void SharedModel::ensureStencils(bool half) {
    if (!stencilLevels) return;
    ensureActiveLists();
    std::lock_guard<std::mutex> g(listMu);
    bool built = false;
    for (size_t l = 1; l < L.size() && l < 63; l++) {
        DevLevel& D = L[l];
        const int cnt = D.useTiles ? (D.split32 ? D.nBnd : 0) : nAct[l];
        if (!((stencilLevels >> l) & 1) || cnt <= 0 || cnt < stencilMinNodes) continue;
        D.stnNodes = D.useTiles ? D.blist.as<int>() : act[l].as<int>();
        D.nStn = cnt;
        const int grid = gridFor(int64_t(cnt) * 27, 256, smCount * 32);
        if (!half && !D.stn32.p) {
            D.stn32.alloc(size_t(cnt) * dev::stnChunks<4>() * 4 * sizeof(float), bytes, ms);
            dev::k_stn_build<float, float><<<grid, 256, 0, ms>>>(D.view, D.c32, D.stnNodes, cnt, D.stn32.as<float>(), 1.f);
            check(cudaGetLastError(), "stencil build");
            built = true;
        }
        if (half && !D.stn16.p) {
            // a bound on every coefficient (at most 8 voxels add to one): 8 x the largest element
            // entry (own matrices below 2^14 hs; s Kb; the diagonal shift), kept below 2^14
            const HostLevel& h = H.levels[l];
            double emax = D.hasOwn ? 16384.0 * double(D.view.hs) : 0.0, kb = 0.0, smax = 0.0, dmax = 0.0;
            for (int e = 0; e < 576; e++) kb = std::max(kb, double(std::fabs(D.c32.Kb[e])));
            for (uint32_t w : h.word)
                if (w && !(w & OWN_BIT)) {
                    float sv;
                    std::memcpy(&sv, &w, sizeof sv);
                    smax = std::max(smax, double(std::fabs(sv)));
                }
            for (double v : h.diagAdd) dmax = std::max(dmax, std::fabs(v));
            const double bound = 8.0 * std::max(emax, smax * kb) + dmax;
            D.stnScale = bound > 0 ? float(std::exp2(std::ceil(std::log2(bound / 16384.0)))) : 1.f;
            D.stn16.alloc(size_t(cnt) * dev::stnChunks<8>() * 8 * sizeof(__half), bytes, ms);
            dev::k_stn_build<__half, float><<<grid, 256, 0, ms>>>(D.view, D.c32, D.stnNodes, cnt, D.stn16.as<__half>(), 1.f / D.stnScale);
            check(cudaGetLastError(), "stencil build");
            built = true;
        }
    }
    if (built) check(cudaEventRecord(readyEv, ms), "event");
}

void SharedModel::ensureBlockStencils() {
    if (!blockStencils) return;
    std::lock_guard<std::mutex> g(listMu);
    if (!bstn32.empty()) return;
    bstn32.resize(L.size());
    for (size_t l = 0; l < L.size(); l++) {
        DevLevel& D = L[l];
        const int cnt = nAct[l];
        if (!cnt) continue;
        const int grid = gridFor(int64_t(cnt) * 27, 256, smCount * 32);
        if (l > 0 || blockStencil0) {
            bstn32[l].alloc(size_t(cnt) * dev::STN_ROW * sizeof(float), bytes, ms);
            dev::k_stn_build<float, float, true><<<grid, 256, 0, ms>>>(D.view, D.c32, act[l].as<int>(), cnt, bstn32[l].as<float>(), 1.f);
            check(cudaGetLastError(), "block stencil build");
        }
    }
    check(cudaEventRecord(readyEv, ms), "event");
}

void SharedModel::ensureActiveLists() {
    std::lock_guard<std::mutex> g(listMu);
    if (!act.empty()) return;
    act.reserve(L.size());
    nAct.resize(L.size());
    for (size_t l = 0; l < L.size(); l++) {
        const HostLevel& h = H.levels[l];
        const int PX = pitch4(h.NX);
        std::vector<int32_t> list;
        for (int64_t row = 0; row < int64_t(h.NY) * h.NZ; row++) {
            const uint8_t* mk = h.nmask.data() + row * h.NX;
            for (int i = 0; i < h.NX; i++)
                if (mk[i] & NM_ACTIVE) list.push_back(int32_t(i + int64_t(PX) * row));
        }
        if (int64_t(PX) * h.NY * h.NZ > int64_t(INT32_MAX)) throw Error(PS_EINVAL, "level too large for 32-bit node lists");
        act.emplace_back();
        nAct[l] = int(list.size());
        upload(act.back(), list, bytes, ms);
    }
    if (const char* e = std::getenv("PSFEA_BLOCK_TC")) blockTc = std::atoi(e) != 0;
    const HostLevel& h0 = H.levels[0];
    if (h0.nOwn == 0) {
        const int ex = (h0.NX + dev::BT_X - 1) / dev::BT_X, ey = (h0.NY + dev::BT_Y - 1) / dev::BT_Y, ez = (h0.NZ + dev::BT_Z - 1) / dev::BT_Z;
        if (ex <= 2047 && ey <= 2047 && ez <= 1023) {
            std::vector<uint8_t> ea(size_t(ex) * ey * ez, 0);
            for (int k = 0; k < h0.NZ; k++)
                for (int j = 0; j < h0.NY; j++) {
                    const uint8_t* row = h0.nmask.data() + h0.node(0, j, k);
                    for (int i = 0; i < h0.NX; i++)
                        if (row[i] & NM_ACTIVE) ea[size_t((i / dev::BT_X) + ex * ((j / dev::BT_Y) + size_t(ey) * (k / dev::BT_Z)))] = 1;
                }
            std::vector<uint32_t> tl;
            for (int tz = 0; tz < ez; tz++)
                for (int ty = 0; ty < ey; ty++)
                    for (int tx = 0; tx < ex; tx++)
                        if (ea[size_t(tx + ex * (ty + size_t(ey) * tz))]) tl.push_back(dev::packTile(tx, ty, tz));
            nBtTiles = int(tl.size());
            upload(btTiles, tl, bytes, ms);
        }
    }
    actReady.store(true, std::memory_order_release);
    check(cudaEventRecord(readyEv, ms), "event");
}

// One solve context: work vectors, control state, stream and recorded iteration graphs over a
// shared hierarchy. A handle has one; concurrent batch solves add more.
struct SolverImpl {
    std::shared_ptr<SharedModel> M;
    Hierarchy& H;
    std::vector<DevLevel>& L;
    DevMem& cDof;
    DevMem& cInv;
    const int& m;
    int smCount;
    std::vector<LevelWork> W;
    // finest-level FP64 work vectors and FP32 mixed-precision ones
    DevMem f, x, r, p, q, z64, x32, p32, q32;
    // control
    DevMem state, partials, ticket;
    int64_t bytes = 0;
    dev::SolveState* hostState = nullptr;  // pinned mirror
    cudaStream_t stream = nullptr;      // the stream every kernel goes to (own, or the caller's)
    cudaStream_t ownStream = nullptr;
    cudaEvent_t ev = nullptr;           // recorded after each asynchronous state read
    int64_t launches = 0;     // kernels launched by this context (graph replays add their kernel count)
    // graphs of one iteration, per precision, and the coefficient version they were recorded with
    // (by ps_precision: FP64 Krylov with the FP32 or the FP16-matrix V-cycle, FP32 Krylov)
    cudaGraphExec_t graph[4] = {nullptr, nullptr, nullptr, nullptr};
    int64_t graphKernels[4] = {0, 0, 0, 0};
    int64_t graphVersion[4] = {-1, -1, -1, -1};
    // the FP32-Krylov forms' fold runs in a conditional branch of the iteration graph (captured on
    // the side stream): foldKernels of them per fold
    cudaStream_t sideStream = nullptr;
    int64_t foldKernels = 0;

    // smoother estimation in flight: its scratch (stream-ordered, freed as soon as the kernels
    // have run) and the Lanczos scalars of every level, copied to pinned host memory
    double* lzHost = nullptr;  // [12 levels][20]
    bool lzPending = false;

    // the solve in progress (a resumable state machine, so one host thread can drive many)
    struct Pending {
        bool active = false, finishing = false, mixed = false, lanczos = false, half = false;
        int graph = 0;  // the iteration graph in use
        const double* fDev = nullptr;
        const double* x0Dev = nullptr;
        ps_solve_opts o{};
        double* uDev = nullptr;
        double* uHost = nullptr;
        std::chrono::steady_clock::time_point t0;
        int batch = 2;
        double lastRel = 0;
        int lastIt = 0;
        ps_status outcome = PS_OK;
        int64_t launches0 = 0;
    } pend;

    explicit SolverImpl(std::shared_ptr<SharedModel> model)
        : M(std::move(model)), H(M->H), L(M->L), cDof(M->cDof), cInv(M->cInv), m(M->m), smCount(M->smCount) {}
    void allocate();

    template <class... KArgs, class... Args>
    void launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args&&... args) {
        kernel<<<grid, block, smem, s>>>(std::forward<Args>(args)...);
        ++launches;
    }

    int nodeGrid(int64_t nNodes) const { return gridFor(nNodes, dev::NODE_THREADS, smCount * 16); }
    // node and DOF counts of level l in the pitched device layout (every device vector's length)
    int64_t pn(int l) const { return L[size_t(l)].view.nNodes; }
    int64_t pd(int l) const { return 3 * pn(l); }
    // tensor maps by (base, kind, level); a base address can only be reused for the same level's
    // vector of the same kind, which has the same map
    std::map<std::tuple<const void*, int, int>, CUtensorMap> mapCache;
    const CUtensorMap& mapOf(const void* base, MapKind kind, bool f64, int l) {
        const auto key = std::make_tuple(base, int(kind) * 2 + (f64 ? 1 : 0), l);
        auto it = mapCache.find(key);
        if (it == mapCache.end()) it = mapCache.emplace(key, makeMap(base, kind, f64, L[size_t(l)].view)).first;
        return it->second;
    }
    // dense reference layout <-> pitched device layout of a level-l DOF vector (device to device)
    void pitch(const double* src, double* dst, int l, bool toPitched) {
        const dev::LevelView& v = L[size_t(l)].view;
        launch(dev::k_pitch<double>, vecGrid(int64_t(v.NX) * v.NY * v.NZ * 3), dev::VEC_THREADS, 0, stream, src, dst, 3, v.NX, v.NY, v.NZ, v.PX,
               toPitched ? 1 : 0);
    }
    // host dense vector -> pitched device vector, through `staging` (a device vector of at least the
    // level's pitched size that holds nothing needed)
    void uploadPitched(const double* host, double* dst, int l, double* staging) {
        const size_t n = size_t(H.levels[size_t(l)].nDof);
        check(cudaMemcpyAsync(staging, host, n * 8, cudaMemcpyHostToDevice, stream), "upload");
        pitch(staging, dst, l, true);
    }
    void downloadPitched(const double* src, double* host, int l, double* staging) {
        const size_t n = size_t(H.levels[size_t(l)].nDof);
        pitch(src, staging, l, false);
        check(cudaMemcpyAsync(host, staging, n * 8, cudaMemcpyDeviceToHost, stream), "download");
    }
    int vecGrid(int64_t n) const { return gridFor(n, dev::VEC_THREADS, smCount * 8); }
    // level l's active-node list when the model has made them (the prolongation's work list)
    // the V-cycle being recorded reads the FP16 stencils (the FP32-Krylov forms)
    bool stn16Pass = false;
    // (only once this context's stream has waited for the lists' upload)
    const int* fineList(int l) const { return listsWaited ? M->act[size_t(l)].as<int>() : nullptr; }
    bool listsWaited = false;
    dev::SolveState* st() const { return state.as<dev::SolveState>(); }
    double* part() const { return partials.as<double>(); }
    unsigned* tick() const { return ticket.as<unsigned>(); }

    void prepareSmoothers();
    void setDegree(int want) {
        if (want == M->degree) return;
        M->degree = want;
        M->smoothersReady = false;
    }
    void enqueueLanczos(int l);       // 10 Lanczos steps of level l, scalars to lzHost[l]
    bool enqueueAllLanczos();         // every level without an estimate; false if none
    void finishLanczos();             // lmax of those levels from lzHost (after the event)
    void computeCoefficients();
    void startIterations();

    // operator launches
    void op64(int l, const double* x, double* y, bool raw, dev::Ctl ctl);
    template <int MODE>
    void op32(int l, const float* x, float* y, float c1, float c2, dev::Ctl ctl, bool own16 = false);
    // V-cycle on level l from W[l].r; returns the buffer holding the result
    // firstDone: W[l].d and W[l].z already hold the first smoothing step (fused upstream)
    float* vcycle(int l, dev::Ctl ctl, bool own16, bool firstDone = false);
    // PS_PREC_HALF: level l >= 1 over its active-node list on FP16 vectors; the V-cycle with FP16
    // vectors below the finest level (vcycleHalf: level 0, FP32; vcycle16: levels >= 1)
    template <int MODE>
    void op16(int l, const __half* x, __half* y, float c1, float c2, dev::Ctl ctl, bool own16);
    float* vcycleHalf(dev::Ctl ctl, bool own16, bool firstDone);
    __half* vcycle16(int l, dev::Ctl ctl, bool own16, bool firstDone);
    float* vcycleFor(bool half, dev::Ctl ctl, bool own16, bool firstDone = false) {
        return half ? vcycleHalf(ctl, own16, firstDone) : vcycle(0, ctl, own16, firstDone);
    }
    bool exactOneLevel() const { return M->exactOneLevel(); }

    void recordPlainIteration(dev::Ctl ctl, bool own16);
    void recordMixedIteration(dev::Ctl ctl, bool refine, bool half);
    // enqueue a solve (f, x0, u in device memory; uHost, if set, receives u as well)
    void startSolve(const double* fDev, const double* x0Dev, const ps_solve_opts& o, double* uDev, double* uHost);
    // move the solve on; returns true (and fills res) once it has finished. block: wait for the
    // GPU instead of returning when it is still busy.
    bool advance(bool block, ps_solve_result& res);
    ps_status runSolve(const double* fDev, const double* x0Dev, const ps_solve_opts& o, double* uDev, ps_solve_result& res) {
        startSolve(fDev, x0Dev, o, uDev, nullptr);
        while (!advance(true, res)) {
        }
        return ps_status(res.status);
    }
    void enqueueStateRead() {
        check(cudaMemcpyAsync(hostState, state.p, sizeof(dev::SolveState), cudaMemcpyDeviceToHost, stream), "state read");
        check(cudaEventRecord(ev, stream), "event");
    }
    void readState() {
        enqueueStateRead();
        check(cudaEventSynchronize(ev), "sync");
    }

    ~SolverImpl() {
        // a caller's stream (setStream) may already be gone: wait for this context's own one only
        if (ownStream) cudaStreamSynchronize(ownStream);
        for (auto& g : graph)
            if (g) cudaGraphExecDestroy(g);
        for (auto& w : W) w.release();
        for (DevMem* b : {&f, &x, &r, &p, &q, &z64, &x32, &p32, &q32, &state, &partials, &ticket}) b->release();
        if (ev) cudaEventDestroy(ev);
        if (sideStream) cudaStreamDestroy(sideStream);
        if (hostState) cudaFreeHost(hostState);
        if (lzHost) cudaFreeHost(lzHost);
        if (ownStream) {
            cudaStreamSynchronize(ownStream);
            cudaStreamDestroy(ownStream);
        }
    }
};

void SolverImpl::allocate() {
    check(cudaStreamCreateWithFlags(&ownStream, cudaStreamNonBlocking), "stream");
    stream = ownStream;
    check(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "event");
    check(cudaMallocHost(&hostState, sizeof(dev::SolveState)), "cudaMallocHost");
    check(cudaMallocHost(&lzHost, 12 * 20 * sizeof(double)), "cudaMallocHost");
    cudaStream_t s = ownStream;
    W.resize(H.levels.size());
    for (size_t l = 0; l < W.size(); l++) {
        const size_t n = size_t(pd(int(l)));
        W[l].r.alloc(n * 4, bytes, s);
        W[l].z.alloc(n * 4, bytes, s);
        W[l].t.alloc(n * 4, bytes, s);
        W[l].d.alloc(n * 4, bytes, s);
    }
    const size_t n = size_t(pd(0));
    f.alloc(n * 8, bytes, s);
    x.alloc(n * 8, bytes, s);
    r.alloc(n * 8, bytes, s);
    p.alloc(n * 8, bytes, s);
    q.alloc(n * 8, bytes, s);
    if (exactOneLevel()) z64.alloc(n * 8, bytes, s);
    x32.alloc(n * 4, bytes, s);
    p32.alloc(n * 4, bytes, s);
    q32.alloc(n * 4, bytes, s);
    state.alloc(sizeof(dev::SolveState), bytes, s);
    partials.alloc(size_t(std::max(smCount * 16, M->maxTiles)) * 4 * sizeof(double) + 4096, bytes, s);
    ticket.alloc(64, bytes, s);
    // the shared data is uploaded on the model's stream: this context's work starts after it
    check(cudaStreamWaitEvent(s, M->readyEv, 0), "wait");
}

void SolverImpl::op64(int l, const double* xin, double* y, bool raw, dev::Ctl ctl) {
    DevLevel& D = L[size_t(l)];
    if (!D.nTiles) return;
    if (!D.useTiles) {
        if (D.use8)
            launch(dev::k_op8<double, dev::OP_APPLY, false, false>, gridFor(D.view.nNodes * 8, 256, smCount * 32), 256, 0, stream, D.view, D.c64, xin,
                   y, nullptr, nullptr, 0.f, 0.f, raw ? 1 : 0, ctl);
        else
            launch(dev::k_op<double, dev::OP_APPLY, false>, nodeGrid(D.view.nNodes), dev::NODE_THREADS, 0, stream, D.view, D.c64, xin, y, nullptr,
                   nullptr, 0.f, 0.f, raw ? 1 : 0, ctl);
        return;
    }
    dev::TileIO<double> io{0.f, 0.f, raw ? 1 : 0, 0};
    dev::TileMaps mp;
    mp.x = mapOf(xin, MAP_HALO, true, l);
    mp.w = mapOf(D.word.p, MAP_WORDS, false, l);
    mp.y = mapOf(y, MAP_TILE, true, l);
    mp.r = mp.d = mp.inv = mp.y;  // not read by this epilogue
    if (D.inner64) {
        launch(dev::k_tile<double, dev::TOP_APPLY, false, false, true>, D.nTiles, dev::TILE_THREADS, dev::tileSmemBytes<double, dev::TOP_APPLY, true>(),
               stream, D.view, D.c64, D.tiles.as<uint32_t>(), mp, io, st(), part(), tick(), ctl);
        return;
    }
    launch(dev::k_tile<double, dev::TOP_APPLY, false, false>, D.nTiles, dev::TILE_THREADS, dev::tileSmemBytes<double, dev::TOP_APPLY, false>(), stream,
           D.view, D.c64, D.tiles.as<uint32_t>(), mp, io, st(), part(), tick(), ctl);
    if (D.nBnd)
        launch(dev::k_bnd<double, dev::TOP_APPLY, false, false>, nodeGrid(D.nBnd), dev::NODE_THREADS, 0, stream, D.view, D.c64,
               D.blist.as<int>(), D.nBnd, xin, y, nullptr, nullptr, 0.f, 0.f, raw ? 1 : 0, st(), part(), tick(), ctl);
}

template <int MODE>
void SolverImpl::op32(int l, const float* xin, float* y, float c1, float c2, dev::Ctl ctl, bool own16) {
    DevLevel& D = L[size_t(l)];
    if (!D.nTiles) return;
    float* rr = W[size_t(l)].r.as<float>();
    float* dd = W[size_t(l)].d.as<float>();
    if (own16 && D.ebe) {
        // the reduced-precision forms: the element-block product on the tensor cores
        constexpr int EM = MODE == dev::OP_CHEB ? dev::TOP_CHEB : (MODE == dev::OP_RESID ? dev::TOP_RESID : dev::TOP_APPLY);
        const uint32_t* et = D.ebeTiles.as<uint32_t>();
        if (M->ebeSplit == 1)
            launch(dev::k_ebe<EM, 1>, D.nEbeTiles, dev::EBE_THREADS, dev::ebeSmemBytes<1>(), stream, D.view, static_cast<const dev::Coefs<float>&>(D.c32),
                   et, xin, y, rr, dd, c1, c2, 0, st(), ctl);
        else
            launch(dev::k_ebe<EM, 3>, D.nEbeTiles, dev::EBE_THREADS, dev::ebeSmemBytes<3>(), stream, D.view, static_cast<const dev::Coefs<float>&>(D.c32),
                   et, xin, y, rr, dd, c1, c2, 0, st(), ctl);
        return;
    }
    const bool o16 = own16 && D.hasOwn, diff = o16 && M->ownDiff;
    constexpr int SM_ = MODE == dev::OP_CHEB ? dev::TOP_CHEB : (MODE == dev::OP_RESID ? dev::TOP_RESID : dev::TOP_APPLY);
    // the assembled stencils of the listed nodes: FP16 in the FP32-Krylov forms, FP32 in the
    // FP64-Krylov ones (PS_PREC_MIXED included: FP16 rounding of the assembled sums, the uniformly
    // scaled voxels' exact FP32 part included, moved its iteration count on the ill-conditioned
    // L-bracket at rel. res. 1e-11 from the reference's 3015 to 3501)
    const bool s16 = o16 && stn16Pass;
    auto stencilPass = [&]() {
        const int g = gridFor(D.nStn, 256, smCount * 16);
        if (s16)
            launch(dev::k_stn<SM_, __half, float>, g, 256, 0, stream, D.view, D.stnNodes, D.nStn, D.stn16.as<__half>(), D.stnScale, xin, y, rr, dd,
                   c1, c2, 1.f, 0, ctl);
        else
            launch(dev::k_stn<SM_, float, float>, g, 256, 0, stream, D.view, D.stnNodes, D.nStn, D.stn32.as<float>(), 1.f, xin, y, rr, dd, c1, c2,
                   1.f, 0, ctl);
    };
    const bool stn = l > 0 && !diff && D.nStn > 0 && (s16 ? D.stn16.p != nullptr : D.stn32.p != nullptr);
    if (stn && !D.useTiles) {
        stencilPass();
        return;
    }
    if (l < 63 && ((M->listLevels >> l) & 1) && !diff && !M->act.empty()) {
        // the whole level over its active-node list
        constexpr int LM = MODE == dev::OP_CHEB ? dev::TOP_CHEB : (MODE == dev::OP_RESID ? dev::TOP_RESID : dev::TOP_APPLY);
        const int* al = M->act[size_t(l)].as<int>();
        const int na = M->nAct[size_t(l)];
        const size_t cls = D.hasOwn ? size_t(D.nOwnDev) * 576 * (o16 ? 2 : 4) : 0;
        if (D.hasOwn && cls <= M->clsSmemMax) {
            const int gc = std::min(smCount, (na + 511) / 512);
            if (o16) launch(dev::k_list<LM, true, true>, gc, 512, cls, stream, D.view, static_cast<const dev::Coefs<float>&>(D.c32), al, na, D.nOwnDev, xin, y, rr, dd, c1, c2, 1.f, 0, ctl);
            else launch(dev::k_list<LM, false, true>, gc, 512, cls, stream, D.view, static_cast<const dev::Coefs<float>&>(D.c32), al, na, D.nOwnDev, xin, y, rr, dd, c1, c2, 1.f, 0, ctl);
        } else {
            const int gl = gridFor(na, 512, smCount * 2);
            if (o16) launch(dev::k_list<LM, true, false>, gl, 512, 0, stream, D.view, static_cast<const dev::Coefs<float>&>(D.c32), al, na, 0, xin, y, rr, dd, c1, c2, 1.f, 0, ctl);
            else launch(dev::k_list<LM, false, false>, gl, 512, 0, stream, D.view, static_cast<const dev::Coefs<float>&>(D.c32), al, na, 0, xin, y, rr, dd, c1, c2, 1.f, 0, ctl);
        }
        return;
    }
    if (D.use8) {
        const int g = gridFor(D.view.nNodes * 8, 256, smCount * 32);
        if (diff) launch(dev::k_op8<float, MODE, true, true>, g, 256, 0, stream, D.view, D.c32, xin, y, rr, dd, c1, c2, 0, ctl);
        else if (o16) launch(dev::k_op8<float, MODE, true, false>, g, 256, 0, stream, D.view, D.c32, xin, y, rr, dd, c1, c2, 0, ctl);
        else launch(dev::k_op8<float, MODE, false, false>, g, 256, 0, stream, D.view, D.c32, xin, y, rr, dd, c1, c2, 0, ctl);
        return;
    }
    if (!D.useTiles) {
        const int g = nodeGrid(D.view.nNodes);
        if (diff) launch(dev::k_op<float, MODE, true, true>, g, dev::NODE_THREADS, 0, stream, D.view, D.c32, xin, y, rr, dd, c1, c2, 0, ctl);
        else if (o16) launch(dev::k_op<float, MODE, true>, g, dev::NODE_THREADS, 0, stream, D.view, D.c32, xin, y, rr, dd, c1, c2, 0, ctl);
        else launch(dev::k_op<float, MODE, false>, g, dev::NODE_THREADS, 0, stream, D.view, D.c32, xin, y, rr, dd, c1, c2, 0, ctl);
        return;
    }
    constexpr int TM = MODE == dev::OP_CHEB ? dev::TOP_CHEB : (MODE == dev::OP_RESID ? dev::TOP_RESID : dev::TOP_APPLY);
    dev::TileIO<float> io{c1, c2, 0, 0};
    dev::TileMaps mp;
    mp.x = mapOf(xin, MAP_HALO, false, l);
    mp.w = mapOf(D.word.p, MAP_WORDS, false, l);
    mp.y = mapOf(y, MAP_TILE, false, l);
    mp.r = dev::tileHasR(TM) ? mapOf(rr, MAP_TILE, false, l) : mp.y;
    mp.d = dev::tileHasD(TM) ? mapOf(dd, MAP_TILE, false, l) : mp.y;
    mp.inv = dev::tileHasD(TM) ? mapOf(D.invD.p, MAP_TILE, false, l) : mp.y;
    const uint32_t* tl = D.tiles.as<uint32_t>();
    if (D.split32) {
        // uniform nodes in the tiles, boundary nodes from the list at full occupancy (the tiles
        // store a boundary node's staged d unchanged, and k_bnd overwrites its d and y)
        const size_t sm = dev::tileSmemBytes<float, TM, false>();
        const dev::Coefs<float>& c = D.c32;
        if (diff) launch(dev::k_tile<float, TM, true, true, false>, D.nTiles, dev::TILE_THREADS, sm, stream, D.view, D.c32, tl, mp, io, st(), part(), tick(), ctl);
        else if (o16) launch(dev::k_tile<float, TM, true, false, false>, D.nTiles, dev::TILE_THREADS, sm, stream, D.view, D.c32, tl, mp, io, st(), part(), tick(), ctl);
        else launch(dev::k_tile<float, TM, false, false, false>, D.nTiles, dev::TILE_THREADS, sm, stream, D.view, D.c32, tl, mp, io, st(), part(), tick(), ctl);
        if (!D.nBnd) return;
        if (stn) {
            stencilPass();
            return;
        }
        const int* bl = D.blist.as<int>();
        if (!diff && D.hasOwn) {
            // few Galerkin classes: the boundary pass gathers from a shared-memory copy of them
            const size_t cls = size_t(D.nOwnDev) * 576 * (o16 ? 2 : 4);
            if (cls <= M->clsSmemMax) {
                const int gc = std::min(smCount, (D.nBnd + 511) / 512);
                if (o16) launch(dev::k_list<TM, true, true>, gc, 512, cls, stream, D.view, c, bl, D.nBnd, D.nOwnDev, xin, y, rr, dd, c1, c2, 1.f, 0, ctl);
                else launch(dev::k_list<TM, false, true>, gc, 512, cls, stream, D.view, c, bl, D.nBnd, D.nOwnDev, xin, y, rr, dd, c1, c2, 1.f, 0, ctl);
                return;
            }
        }
        const int g = gridFor(D.nBnd, dev::NODE_THREADS, smCount * 16);
        if (diff) launch(dev::k_bnd<float, TM, true, true>, g, dev::NODE_THREADS, 0, stream, D.view, c, bl, D.nBnd, xin, y, rr, dd, c1, c2, 0, st(), part(), tick(), ctl);
        else if (o16) launch(dev::k_bnd<float, TM, true, false>, g, dev::NODE_THREADS, 0, stream, D.view, c, bl, D.nBnd, xin, y, rr, dd, c1, c2, 0, st(), part(), tick(), ctl);
        else launch(dev::k_bnd<float, TM, false, false>, g, dev::NODE_THREADS, 0, stream, D.view, c, bl, D.nBnd, xin, y, rr, dd, c1, c2, 0, st(), part(), tick(), ctl);
        return;
    }
    const size_t sm = dev::tileSmemBytes<float, TM, true>();
    if (diff) launch(dev::k_tile<float, TM, true, true>, D.nTiles, dev::TILE_THREADS, sm, stream, D.view, D.c32, tl, mp, io, st(), part(), tick(), ctl);
    else if (o16) launch(dev::k_tile<float, TM, true, false>, D.nTiles, dev::TILE_THREADS, sm, stream, D.view, D.c32, tl, mp, io, st(), part(), tick(), ctl);
    else launch(dev::k_tile<float, TM, false, false>, D.nTiles, dev::TILE_THREADS, sm, stream, D.view, D.c32, tl, mp, io, st(), part(), tick(), ctl);
}

// pre-smoothing from zero, residual, restriction, coarse correction, prolongation, post-smoothing
// (voxel_fea.cpp:817-828); buffers alternate between the level's z and t
float* SolverImpl::vcycle(int l, dev::Ctl ctl, bool own16, bool firstDone) {
    DevLevel& D = L[size_t(l)];
    const HostLevel& h = H.levels[size_t(l)];
    LevelWork& Wl = W[size_t(l)];
    float *z = Wl.z.as<float>(), *t = Wl.t.as<float>(), *r = Wl.r.as<float>(), *d = Wl.d.as<float>();
    const int last = int(L.size()) - 1;
    if (l == last) {
        if (H.hasFactor()) {
            const int threads = 256, warps = threads / 32;
            const int grid = std::max(1, std::min(smCount * 2, (m + warps - 1) / warps));
            launch(dev::k_coarse<float, float>, grid, threads, size_t(m) * sizeof(double), stream, m, cDof.as<int>(), cInv.as<double>(), r, z, 1.0, ctl);
            return z;
        }
        // no factor: 40 damped Jacobi sweeps with the default weight (voxel_fea.cpp:676-678)
        if (!firstDone)
            launch(dev::k_cheb_first<float>, vecGrid(pd(l)), dev::VEC_THREADS, 0, stream, pd(l), r, D.invD.as<float>(), d, z, D.omega, ctl);
        float* a = z;
        float* b = t;
        for (int s = 1; s < 40; s++) {
            op32<dev::OP_CHEB>(l, a, b, 0.f, D.omega, ctl, own16);
            std::swap(a, b);
        }
        return a;
    }
    DevLevel& C = L[size_t(l + 1)];
    LevelWork& Wc = W[size_t(l + 1)];
    const HostLevel& hc = H.levels[size_t(l + 1)];
    if (!firstDone)
        launch(dev::k_cheb_first<float>, vecGrid(pd(l)), dev::VEC_THREADS, 0, stream, pd(l), r, D.invD.as<float>(), d, z, D.cf0, ctl);
    float* a = z;  // the current iterate
    float* b = t;
    for (size_t k = 0; k < D.chebC1.size(); k++) {  // pre-smoothing from zero
        op32<dev::OP_CHEB>(l, a, b, D.chebC1[k], D.chebC2[k], ctl, own16);
        std::swap(a, b);
    }
    op32<dev::OP_RESID>(l, a, b, 0.f, 0.f, ctl, own16);  // b = r - K a
    // restriction, with the coarse level's first smoothing step fused in (unless it is the dense solve)
    const bool fuse = !(l + 1 == last && H.hasFactor());
    const float c0c = (l + 1 == last) ? C.omega : C.cf0;
    launch(dev::k_restrict<float, float>, gridFor(pn(l + 1), 256, smCount * 16), 256, 0, stream, D.view, C.view, b, Wc.r.as<float>(),
           fuse ? Wc.d.as<float>() : nullptr, fuse ? Wc.z.as<float>() : nullptr, c0c, 1.f, ctl);
    float* zc = vcycle(l + 1, ctl, own16, fuse);
    {
        const int* pl = fineList(l);
        const int64_t pc = pl ? M->nAct[size_t(l)] : pn(l);
        launch(dev::k_prolong<float, float>, gridFor(pc, 256, smCount * 16), 256, 0, stream, D.view, C.view.PX, hc.NY, pl, (long long)pc, zc, a,
               1.f, ctl);
    }
    op32<dev::OP_CHEB>(l, a, b, 0.f, D.cf0, ctl, own16);  // post-smoothing: d = c0 D^-1 (r - K a); b = a + d
    std::swap(a, b);
    for (size_t k = 0; k < D.chebC1.size(); k++) {
        op32<dev::OP_CHEB>(l, a, b, D.chebC1[k], D.chebC2[k], ctl, own16);
        std::swap(a, b);
    }
    return a;
}

template <int MODE>
void SolverImpl::op16(int l, const __half* xin, __half* y, float c1, float c2, dev::Ctl ctl, bool own16) {
    DevLevel& D = L[size_t(l)];
    const int na = M->nAct[size_t(l)];
    if (!na) return;
    constexpr int LM = MODE == dev::OP_CHEB ? dev::TOP_CHEB : (MODE == dev::OP_RESID ? dev::TOP_RESID : dev::TOP_APPLY);
    const float delta = M->halfDelta[size_t(l)], rho = 1.f / delta;
    const __half* rr = W[size_t(l)].r.as<__half>();
    __half* dd = W[size_t(l)].d.as<__half>();
    const int* al = M->act[size_t(l)].as<int>();
    const bool o16 = own16 && D.hasOwn;
    const dev::Coefs<float>& c = D.c32;
    const size_t cls = D.hasOwn ? size_t(D.nOwnDev) * 576 * (o16 ? 2 : 4) : 0;
    if (D.hasOwn && cls <= M->clsSmemMax) {
        const int gc = std::min(smCount, (na + 511) / 512);
        if (o16) launch(dev::k_list<LM, true, true, __half>, gc, 512, cls, stream, D.view, c, al, na, D.nOwnDev, xin, y, rr, dd, c1, c2 * delta, rho, 0, ctl);
        else launch(dev::k_list<LM, false, true, __half>, gc, 512, cls, stream, D.view, c, al, na, D.nOwnDev, xin, y, rr, dd, c1, c2 * delta, rho, 0, ctl);
    } else {
        const int g = gridFor(na, 512, smCount * 2);
        if (o16) launch(dev::k_list<LM, true, false, __half>, g, 512, 0, stream, D.view, c, al, na, 0, xin, y, rr, dd, c1, c2 * delta, rho, 0, ctl);
        else launch(dev::k_list<LM, false, false, __half>, g, 512, 0, stream, D.view, c, al, na, 0, xin, y, rr, dd, c1, c2 * delta, rho, 0, ctl);
    }
}

// The finest level of the FP16 V-cycle: vcycle's level 0 (FP32 vectors), restricting into and
// prolongating from level 1's FP16 vectors (residual scale 1/8 there; iterate scale delta_1 / 8)
float* SolverImpl::vcycleHalf(dev::Ctl ctl, bool own16, bool firstDone) {
    DevLevel& D = L[0];
    LevelWork& W0 = W[0];
    float *z = W0.z.as<float>(), *t = W0.t.as<float>(), *r = W0.r.as<float>(), *d = W0.d.as<float>();
    DevLevel& C = L[1];
    LevelWork& Wc = W[1];
    const HostLevel& hc = H.levels[1];
    const int last = int(L.size()) - 1;
    const float dc = M->halfDelta[1];
    if (!firstDone)
        launch(dev::k_cheb_first<float>, vecGrid(pd(0)), dev::VEC_THREADS, 0, stream, pd(0), r, D.invD.as<float>(), d, z, D.cf0, ctl);
    float* a = z;
    float* b = t;
    for (size_t k = 0; k < D.chebC1.size(); k++) {
        op32<dev::OP_CHEB>(0, a, b, D.chebC1[k], D.chebC2[k], ctl, own16);
        std::swap(a, b);
    }
    op32<dev::OP_RESID>(0, a, b, 0.f, 0.f, ctl, own16);
    const bool fuse = !(1 == last && H.hasFactor());
    const float c0c = (1 == last) ? C.omega : C.cf0;
    launch(dev::k_restrict<float, __half>, gridFor(pn(1), 256, smCount * 16), 256, 0, stream, D.view, C.view, b, Wc.r.as<__half>(),
           fuse ? Wc.d.as<__half>() : nullptr, fuse ? Wc.z.as<__half>() : nullptr, c0c * dc, 0.125f, ctl);
    const __half* zc = vcycle16(1, ctl, own16, fuse);
    {
        const int* pl = fineList(0);
        const int64_t pc = pl ? M->nAct[0] : pn(0);
        launch(dev::k_prolong<__half, float>, gridFor(pc, 256, smCount * 16), 256, 0, stream, D.view, C.view.PX, hc.NY, pl, (long long)pc, zc, a,
               8.f / dc, ctl);
    }
    op32<dev::OP_CHEB>(0, a, b, 0.f, D.cf0, ctl, own16);
    std::swap(a, b);
    for (size_t k = 0; k < D.chebC1.size(); k++) {
        op32<dev::OP_CHEB>(0, a, b, D.chebC1[k], D.chebC2[k], ctl, own16);
        std::swap(a, b);
    }
    return a;
}

// vcycle on level l >= 1 with FP16 vectors (residuals r * 8^-l, iterates x * 8^-l * delta_l)
__half* SolverImpl::vcycle16(int l, dev::Ctl ctl, bool own16, bool firstDone) {
    DevLevel& D = L[size_t(l)];
    LevelWork& Wl = W[size_t(l)];
    __half *z = Wl.z.as<__half>(), *t = Wl.t.as<__half>(), *r = Wl.r.as<__half>(), *d = Wl.d.as<__half>();
    const float dl = M->halfDelta[size_t(l)];
    const int last = int(L.size()) - 1;
    if (l == last) {
        if (H.hasFactor()) {
            const int threads = 256, warps = threads / 32;
            const int grid = std::max(1, std::min(smCount * 2, (m + warps - 1) / warps));
            // held DOFs are not written by the solve and must read 0 (the buffer is shared with
            // the FP32 forms' vectors, laid out differently)
            check(cudaMemsetAsync(z, 0, size_t(pd(l)) * sizeof(__half), stream), "memset");
            launch(dev::k_coarse<__half, __half>, grid, threads, size_t(m) * sizeof(double), stream, m, cDof.as<int>(), cInv.as<double>(), r, z,
                   double(dl), ctl);
            return z;
        }
        if (!firstDone)
            launch(dev::k_cheb_first<__half>, vecGrid(pd(l)), dev::VEC_THREADS, 0, stream, pd(l), r, D.invD.as<float>(), d, z, D.omega * dl, ctl);
        __half* a = z;
        __half* b = t;
        for (int s = 1; s < 40; s++) {
            op16<dev::OP_CHEB>(l, a, b, 0.f, D.omega, ctl, own16);
            std::swap(a, b);
        }
        return a;
    }
    DevLevel& C = L[size_t(l + 1)];
    LevelWork& Wc = W[size_t(l + 1)];
    const HostLevel& hc = H.levels[size_t(l + 1)];
    const float dc = M->halfDelta[size_t(l + 1)];
    if (!firstDone)
        launch(dev::k_cheb_first<__half>, vecGrid(pd(l)), dev::VEC_THREADS, 0, stream, pd(l), r, D.invD.as<float>(), d, z, D.cf0 * dl, ctl);
    __half* a = z;
    __half* b = t;
    for (size_t k = 0; k < D.chebC1.size(); k++) {
        op16<dev::OP_CHEB>(l, a, b, D.chebC1[k], D.chebC2[k], ctl, own16);
        std::swap(a, b);
    }
    op16<dev::OP_RESID>(l, a, b, 0.f, 0.f, ctl, own16);
    const bool fuse = !(l + 1 == last && H.hasFactor());
    const float c0c = (l + 1 == last) ? C.omega : C.cf0;
    launch(dev::k_restrict<__half, __half>, gridFor(pn(l + 1), 256, smCount * 16), 256, 0, stream, D.view, C.view, b, Wc.r.as<__half>(),
           fuse ? Wc.d.as<__half>() : nullptr, fuse ? Wc.z.as<__half>() : nullptr, c0c * dc, 0.125f, ctl);
    const __half* zc = vcycle16(l + 1, ctl, own16, fuse);
    {
        const int* pl = fineList(l);
        const int64_t pc = pl ? M->nAct[size_t(l)] : pn(l);
        launch(dev::k_prolong<__half, __half>, gridFor(pc, 256, smCount * 16), 256, 0, stream, D.view, C.view.PX, hc.NY, pl, (long long)pc, zc, a,
               8.f * dl / dc, ctl);
    }
    op16<dev::OP_CHEB>(l, a, b, 0.f, D.cf0, ctl, own16);
    std::swap(a, b);
    for (size_t k = 0; k < D.chebC1.size(); k++) {
        op16<dev::OP_CHEB>(l, a, b, D.chebC1[k], D.chebC2[k], ctl, own16);
        std::swap(a, b);
    }
    return a;
}

// 10 Lanczos steps on D^-1/2 K D^-1/2 from the reference's LCG start vector (voxel_fea.cpp:579-610),
// all on the device and stream-ordered (scratch freed behind the kernels); the 20 scalars go to
// pinned host memory and finishLanczos applies the reference's stop rule (b <= 1e-12 |a| ends the
// sequence; later steps are ignored)
void SolverImpl::enqueueLanczos(int l) {
    DevLevel& D = L[size_t(l)];
    const HostLevel& h = H.levels[size_t(l)];
    const int64_t n = pd(l);
    int64_t scratch = 0;
    DevMem v, vp, w, xx, invD, ab;
    v.alloc(size_t(n) * 8, scratch, stream);
    vp.alloc(size_t(n) * 8, scratch, stream);
    w.alloc(size_t(n) * 8, scratch, stream);
    xx.alloc(size_t(n) * 8, scratch, stream);
    ab.alloc(20 * sizeof(double), scratch, stream);
    upload(invD, pitched<double>(h.invDiag, 3, h, D.view.PX, 0.0), scratch, stream);
    const int vg = vecGrid(n);
    launch(dev::k_lz_start, nodeGrid(pn(l)), dev::NODE_THREADS, 0, stream, D.view, v.as<double>(), part(), tick(), st());
    launch(dev::k_scale, vg, dev::VEC_THREADS, 0, stream, n, v.as<double>(), st());
    const dev::Ctl none{nullptr, nullptr};
    double* abp = ab.as<double>();
    for (int s = 0; s < 10; s++) {
        launch(dev::k_lz_x, vg, dev::VEC_THREADS, 0, stream, n, invD.as<double>(), v.as<double>(), xx.as<double>());
        op64(l, xx.as<double>(), w.as<double>(), false, none);
        launch(dev::k_lz_w, vg, dev::VEC_THREADS, 0, stream, n, invD.as<double>(), w.as<double>(), v.as<double>(), vp.as<double>(),
               s == 0 ? nullptr : abp + 10 + s - 1, abp + s, st(), part(), tick());
        launch(dev::k_lz_axpy, vg, dev::VEC_THREADS, 0, stream, n, w.as<double>(), v.as<double>(), abp + s, abp + 10 + s, st(), part(), tick());
        launch(dev::k_lz_next, vg, dev::VEC_THREADS, 0, stream, n, w.as<double>(), v.as<double>(), vp.as<double>(), abp + 10 + s);
    }
    check(cudaMemcpyAsync(lzHost + 20 * l, abp, 20 * sizeof(double), cudaMemcpyDeviceToHost, stream), "lanczos read");
    check(cudaGetLastError(), "lanczos");
}  // the scratch buffers are released here, stream-ordered behind the kernels

bool SolverImpl::enqueueAllLanczos() {
    bool any = false;
    for (int l = 0; l + 1 < int(L.size()); l++)
        if (!(H.levels[size_t(l)].lmax > 0)) {
            enqueueLanczos(l);
            any = true;
        }
    if (any) check(cudaEventRecord(ev, stream), "event");
    lzPending = any;
    return any;
}

void SolverImpl::finishLanczos() {
    for (int l = 0; l + 1 < int(L.size()); l++) {
        HostLevel& h = H.levels[size_t(l)];
        if (h.lmax > 0) continue;
        const double* hab = lzHost + 20 * l;
        std::vector<double> alpha, beta;
        for (int s = 0; s < 10; s++) {
            const double a = hab[s], b = hab[10 + s];  // hab[10 + s] holds |w| after step s
            alpha.push_back(a);
            if (!(b > 1e-12 * std::fabs(a))) break;
            beta.push_back(b);
        }
        beta.resize(alpha.size() - 1);
        h.lmax = tridiagonalMax(alpha, beta);
    }
    lzPending = false;
}

void SolverImpl::computeCoefficients() {
    for (int l = 0; l + 1 < int(L.size()); l++) {
        HostLevel& h = H.levels[size_t(l)];
        DevLevel& D = L[size_t(l)];
        double c0, c1, c2;
        chebyshevCoefficients(h.lmax, c0, c1, c2);
        D.cf0 = float(c0);
        D.cf1 = float(c1);
        D.cf2 = float(c2);
        D.omega = float(1.2 / (h.lmax * 1.05));
        // the Chebyshev recurrence on [0.1, 1.15] lmax continued to `degree` steps (Adams et al.
        // 2003); step 1 is the reference's second step (voxel_fea.cpp:692-701)
        const double b = 1.15 * h.lmax, a = 0.1 * h.lmax, theta = (b + a) / 2, delta = (b - a) / 2, sigma = theta / delta;
        double rho = 1 / sigma;
        D.chebC1.clear();
        D.chebC2.clear();
        for (int k = 1; k < M->degree; k++) {
            const double rn = 1 / (2 * sigma - rho);
            D.chebC1.push_back(float(rn * rho));
            D.chebC2.push_back(float(2 * rn / delta));
            rho = rn;
        }
    }
    // the coarsest level keeps the default Jacobi weight 0.5 (its eigenvalue is never estimated)
    M->smoothersReady = true;
    M->version++;
}

void SolverImpl::prepareSmoothers() {
    if (M->smoothersReady) return;
    if (enqueueAllLanczos()) {
        check(cudaEventSynchronize(ev), "lanczos");
        finishLanczos();
    }
    computeCoefficients();
}

// one FP64 CG iteration (voxel_fea.cpp:901-919)
void SolverImpl::recordPlainIteration(dev::Ctl ctl, bool own16) {
    const HostLevel& h = H.levels[0];
    DevLevel& D = L[0];
    LevelWork& W0 = W[0];
    if (!D.useTiles) {
        launch(dev::k_apply_alpha<double, false>, nodeGrid(pn(0)), dev::NODE_THREADS, 0, stream, D.view, D.c64, p.as<double>(), q.as<double>(),
               st(), part(), tick(), ctl);
    } else {
        dev::TileIO<double> io{0.f, 0.f, 0, (D.nBnd && !D.inner64) ? 1 : 0};
        dev::TileMaps mp;
        mp.x = mapOf(p.p, MAP_HALO, true, 0);
        mp.w = mapOf(D.word.p, MAP_WORDS, false, 0);
        mp.y = mapOf(q.p, MAP_TILE, true, 0);
        mp.r = mp.d = mp.inv = mp.y;
        if (D.inner64)
            launch(dev::k_tile<double, dev::TOP_DOT, false, false, true>, D.nTiles, dev::TILE_THREADS, dev::tileSmemBytes<double, dev::TOP_DOT, true>(),
                   stream, D.view, D.c64, D.tiles.as<uint32_t>(), mp, io, st(), part(), tick(), ctl);
        else
            launch(dev::k_tile<double, dev::TOP_DOT, false, false>, D.nTiles, dev::TILE_THREADS, dev::tileSmemBytes<double, dev::TOP_DOT, false>(),
                   stream, D.view, D.c64, D.tiles.as<uint32_t>(), mp, io, st(), part(), tick(), ctl);
        if (D.nBnd && !D.inner64)
            launch(dev::k_bnd<double, dev::TOP_DOT, false, false>, nodeGrid(D.nBnd), dev::NODE_THREADS, 0, stream, D.view, D.c64,
                   D.blist.as<int>(), D.nBnd, p.as<double>(), q.as<double>(), nullptr, nullptr, 0.f, 0.f, 0, st(), part(), tick(), ctl);
    }
    const bool one = exactOneLevel();
    launch(dev::k_cg_update, vecGrid(pn(0)), dev::VEC_THREADS, 0, stream, pn(0), D.view.nmask, x.as<double>(), r.as<double>(), p.as<double>(),
           q.as<double>(), one ? nullptr : W0.r.as<float>(), D.invD.as<float>(), W0.d.as<float>(), W0.z.as<float>(), D.cf0, st(), part(), tick(),
           ctl);
    float* z32 = nullptr;
    if (one) {
        const int threads = 256, warps = threads / 32;
        const int grid = std::max(1, std::min(smCount * 2, (m + warps - 1) / warps));
        launch(dev::k_coarse<double, double>, grid, threads, size_t(m) * sizeof(double), stream, m, cDof.as<int>(), cInv.as<double>(), r.as<double>(),
               z64.as<double>(), 1.0, ctl);
    } else {
        z32 = vcycle(0, ctl, own16, true);  // r32 and the first smoothing step came with the update
    }
    launch(dev::k_cg_dots, vecGrid(pn(0)), dev::VEC_THREADS, 0, stream, pn(0), D.view.nmask, r.as<double>(), z32, z64.as<double>(),
           q.as<double>(), st(), part(), tick(), ctl);
    launch(dev::k_cg_p, vecGrid(pn(0)), dev::VEC_THREADS, 0, stream, pn(0), D.view.nmask, z32, z64.as<double>(), p.as<double>(), st(), ctl);
}

// one FP32 CG iteration with the FP64 fold (runs only when due)
void SolverImpl::recordMixedIteration(dev::Ctl ctl, bool refine, bool half) {
    const HostLevel& h = H.levels[0];
    DevLevel& D = L[0];
    LevelWork& W0 = W[0];
    const int* foldFlag = &st()->fold;
    if (!D.useTiles) {
        launch(dev::k_apply_alpha<float, true>, nodeGrid(pn(0)), dev::NODE_THREADS, 0, stream, D.view, D.c32, p32.as<float>(), q32.as<float>(),
               st(), part(), tick(), dev::Ctl{ctl.skipIf, nullptr});
    } else {
        dev::TileIO<float> io{0.f, 0.f, 0, 0};
        dev::TileMaps mp;
        mp.x = mapOf(p32.p, MAP_HALO, false, 0);
        mp.w = mapOf(D.word.p, MAP_WORDS, false, 0);
        mp.y = mapOf(q32.p, MAP_TILE, false, 0);
        mp.r = mp.d = mp.inv = mp.y;
        launch(dev::k_tile<float, dev::TOP_DOT, false, true>, D.nTiles, dev::TILE_THREADS, dev::tileSmemBytes<float, dev::TOP_DOT, true>(), stream, D.view,
               D.c32, D.tiles.as<uint32_t>(), mp, io, st(), part(), tick(), dev::Ctl{ctl.skipIf, nullptr});
    }
    // the fold (u += x32, the FP64 defect as the new r32) is due every few iterations only: it sits
    // in a conditional branch that the update kernel opens, so that iterations without it launch
    // none of its kernels (a skipped tiled launch still dispatches all its CTAs)
    // (PSFEA_FOLD_BRANCH=0: the fold's kernels inline, each skipping itself unless due; ncu cannot
    // profile the kernels of a graph with a conditional node)
    const bool branch = M->foldBranch;
    cudaStreamCaptureStatus cs;
    cudaGraph_t cg = nullptr;
    cudaGraphConditionalHandle foldIf = 0;
    if (branch) {
        check(cudaStreamGetCaptureInfo_v3(stream, &cs, nullptr, &cg, nullptr, nullptr, nullptr), "capture info");
        check(cudaGraphConditionalHandleCreate(&foldIf, cg, 0, cudaGraphCondAssignDefault), "conditional handle");
    }
    float* invD0 = D.invD.as<float>();
    float *d0 = W0.d.as<float>(), *z0 = W0.z.as<float>();
    launch(dev::k_mx_update, vecGrid(pn(0)), dev::VEC_THREADS, 0, stream, pn(0), D.view.nmask, x32.as<float>(), W0.r.as<float>(),
           p32.as<float>(), q32.as<float>(), invD0, d0, z0, D.cf0, st(), part(), tick(), foldIf, branch ? 1 : 0, ctl);
    const dev::Ctl foldCtl{ctl.skipIf, foldFlag};
    if (!branch) {
        launch(dev::k_mx_fold1, vecGrid(pd(0)), dev::VEC_THREADS, 0, stream, pd(0), x.as<double>(), x32.as<float>(), st(), foldCtl);
        op64(0, x.as<double>(), q.as<double>(), false, foldCtl);
        launch(dev::k_mx_fold2, vecGrid(pn(0)), dev::VEC_THREADS, 0, stream, pn(0), D.view.nmask, f.as<double>(), q.as<double>(),
               W0.r.as<float>(), invD0, d0, z0, D.cf0, st(), part(), tick(), foldCtl);
        if (refine)
            launch(dev::k_mx_rescale, vecGrid(pd(0)), dev::VEC_THREADS, 0, stream, pd(0), W0.r.as<float>(), invD0, d0, z0, D.cf0, st(),
                   dev::Ctl{ctl.skipIf, &st()->restart});
        foldKernels = 0;
        float* z32 = vcycleFor(half, ctl, M->mixedOwn16, true);
        launch(dev::k_mx_dots, vecGrid(pn(0)), dev::VEC_THREADS, 0, stream, pn(0), D.view.nmask, W0.r.as<float>(), z32, q32.as<float>(), st(),
               part(), tick(), ctl);
        launch(dev::k_mx_p, vecGrid(pn(0)), dev::VEC_THREADS, 0, stream, pn(0), D.view.nmask, z32, p32.as<float>(), st(), ctl);
        return;
    }
    const cudaGraphNode_t* deps = nullptr;
    size_t nDeps = 0;
    check(cudaStreamGetCaptureInfo_v3(stream, &cs, nullptr, &cg, &deps, nullptr, &nDeps), "capture info");
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = foldIf;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t foldNode;
    check(cudaGraphAddNode(&foldNode, cg, deps, nDeps, &cp), "conditional node");
    check(cudaStreamUpdateCaptureDependencies(stream, &foldNode, 1, cudaStreamSetCaptureDependencies), "capture dependencies");
    if (!sideStream) check(cudaStreamCreateWithFlags(&sideStream, cudaStreamNonBlocking), "stream");
    cudaStream_t mainStream = stream;
    stream = sideStream;
    check(cudaStreamBeginCaptureToGraph(stream, cp.conditional.phGraph_out[0], nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal),
          "capture the fold");
    const int64_t before = launches;
    launch(dev::k_mx_fold1, vecGrid(pd(0)), dev::VEC_THREADS, 0, stream, pd(0), x.as<double>(), x32.as<float>(), st(), foldCtl);
    op64(0, x.as<double>(), q.as<double>(), false, foldCtl);
    launch(dev::k_mx_fold2, vecGrid(pn(0)), dev::VEC_THREADS, 0, stream, pn(0), D.view.nmask, f.as<double>(), q.as<double>(),
           W0.r.as<float>(), invD0, d0, z0, D.cf0, st(), part(), tick(), foldCtl);
    if (refine)
        launch(dev::k_mx_rescale, vecGrid(pd(0)), dev::VEC_THREADS, 0, stream, pd(0), W0.r.as<float>(), invD0, d0, z0, D.cf0, st(),
               dev::Ctl{ctl.skipIf, &st()->restart});
    foldKernels = launches - before;
    launches = before;  // counted per fold when the solve reports its kernels
    cudaGraph_t body = nullptr;
    check(cudaStreamEndCapture(stream, &body), "capture the fold");
    stream = mainStream;
    float* z32 = vcycleFor(half, ctl, M->mixedOwn16, true);  // the first smoothing step came with the update or the fold
    launch(dev::k_mx_dots, vecGrid(pn(0)), dev::VEC_THREADS, 0, stream, pn(0), D.view.nmask, W0.r.as<float>(), z32, q32.as<float>(), st(), part(),
           tick(), ctl);
    launch(dev::k_mx_p, vecGrid(pn(0)), dev::VEC_THREADS, 0, stream, pn(0), D.view.nmask, z32, p32.as<float>(), st(), ctl);
}

void SolverImpl::startSolve(const double* fDev, const double* x0Dev, const ps_solve_opts& o, double* uDev, double* uHost) {
    pend = Pending{};
    pend.t0 = std::chrono::steady_clock::now();
    pend.launches0 = launches;
    pend.o = o;
    pend.uDev = uDev;
    pend.uHost = uHost;
    pend.fDev = fDev;
    pend.x0Dev = x0Dev;
    pend.active = true;
    setDegree(o.smoother_degree > 0 ? o.smoother_degree : M->defaultDegree);
    if (!M->smoothersReady) {
        // the smoother bounds first: their scalars come back with an event (advance() waits for it)
        if (enqueueAllLanczos()) {
            pend.lanczos = true;
            return;
        }
        computeCoefficients();
    }
    startIterations();
}

void SolverImpl::startIterations() {
    const double* fDev = pend.fDev;
    const double* x0Dev = pend.x0Dev;
    const ps_solve_opts& o = pend.o;
    const HostLevel& h = H.levels[0];
    DevLevel& D = L[0];
    LevelWork& W0 = W[0];
    // FP32 Krylov (PS_PREC_FP32); the FP64 Krylov forms differ only in the V-cycle's matrices
    const bool refine = o.precision == PS_PREC_HALF && !exactOneLevel();
    const bool half = refine && M->halfOk;
    const bool mixed = (o.precision == PS_PREC_FP32 || refine) && !exactOneLevel();
    const bool own16 = o.precision == PS_PREC_MIXED && M->mixedOwn16;
    pend.mixed = mixed;
    pend.half = half;
    stn16Pass = mixed;
    if (!exactOneLevel()) {
        M->ensureStencils(mixed && M->mixedOwn16);
        const bool ready = M->actReady.load(std::memory_order_acquire);
        check(cudaStreamWaitEvent(stream, M->readyEv, 0), "wait");
        listsWaited = listsWaited || ready;
    }
    if (half) {
        M->ensureActiveLists();
        check(cudaStreamWaitEvent(stream, M->readyEv, 0), "wait");
        // the list kernels write active nodes only: the FP16 views of the levels' second iterate
        // buffers (also the FP32 forms' storage) start from zeros, so that their inactive nodes read 0
        for (size_t l = 1; l < W.size(); l++) check(cudaMemsetAsync(W[l].t.p, 0, size_t(pd(int(l))) * sizeof(__half), stream), "memset");
    }
    const int64_t n = pd(0);
    // state
    dev::SolveState s{};
    s.tol = o.tol;
    s.maxIter = o.max_iter;
    s.first = 1;
    s.mixed = mixed ? 1 : 0;
    s.foldFactor = refine ? M->refineEta : M->foldFactor;
    s.refine = refine ? 1 : 0;
    s.rescale = 1.0;
    *hostState = s;
    check(cudaMemcpyAsync(state.p, hostState, sizeof s, cudaMemcpyHostToDevice, stream), "state");
    if (fDev != f.p) pitch(fDev, f.as<double>(), 0, true);  // a caller's device vector (dense layout)
    launch(dev::k_mask_copy, vecGrid(pn(0)), dev::VEC_THREADS, 0, stream, pn(0), D.view.nmask, x0Dev, x.as<double>());
    // the search direction is only ever written at free DOFs: clear what earlier calls left in it
    // (apply, reactions, stresses and warm starts use it as staging)
    check(cudaMemsetAsync(p.p, 0, size_t(pd(0)) * 8, stream), "memset");
    const dev::Ctl none{nullptr, nullptr};
    const dev::Ctl ctl{&st()->done, nullptr};
    op64(0, x.as<double>(), q.as<double>(), false, none);
    launch(dev::k_cg_init, vecGrid(pn(0)), dev::VEC_THREADS, 0, stream, pn(0), D.view.nmask, f.as<double>(), q.as<double>(), r.as<double>(),
           nullptr, st(), part(), tick());
    // first preconditioned direction
    if (mixed) {
        check(cudaMemsetAsync(x32.p, 0, size_t(n) * 4, stream), "memset");
        launch(dev::k_vc_load, vecGrid(pn(0)), dev::VEC_THREADS, 0, stream, pn(0), D.view.nmask, r.as<double>(), W0.r.as<float>(),
               D.invD.as<float>(), W0.d.as<float>(), W0.z.as<float>(), D.cf0, st(), ctl);
        float* z32 = vcycleFor(half, ctl, M->mixedOwn16, true);
        launch(dev::k_mx_dots, vecGrid(pn(0)), dev::VEC_THREADS, 0, stream, pn(0), D.view.nmask, W0.r.as<float>(), z32, q32.as<float>(), st(),
               part(), tick(), ctl);
        launch(dev::k_mx_p, vecGrid(pn(0)), dev::VEC_THREADS, 0, stream, pn(0), D.view.nmask, z32, p32.as<float>(), st(), ctl);
    } else {
        float* z32 = nullptr;
        if (exactOneLevel()) {
            const int threads = 256, warps = threads / 32;
            const int grid = std::max(1, std::min(smCount * 2, (m + warps - 1) / warps));
            check(cudaMemsetAsync(z64.p, 0, size_t(n) * 8, stream), "memset");
            launch(dev::k_coarse<double, double>, grid, threads, size_t(m) * sizeof(double), stream, m, cDof.as<int>(), cInv.as<double>(),
                   r.as<double>(), z64.as<double>(), 1.0, ctl);
        } else {
            launch(dev::k_vc_load, vecGrid(pn(0)), dev::VEC_THREADS, 0, stream, pn(0), D.view.nmask, r.as<double>(), W0.r.as<float>(),
                   D.invD.as<float>(), W0.d.as<float>(), W0.z.as<float>(), D.cf0, st(), ctl);
            z32 = vcycle(0, ctl, own16, true);
        }
        launch(dev::k_cg_dots, vecGrid(pn(0)), dev::VEC_THREADS, 0, stream, pn(0), D.view.nmask, r.as<double>(), z32, z64.as<double>(),
               q.as<double>(), st(), part(), tick(), ctl);
        launch(dev::k_cg_p, vecGrid(pn(0)), dev::VEC_THREADS, 0, stream, pn(0), D.view.nmask, z32, z64.as<double>(), p.as<double>(), st(),
               ctl);
    }
    launch(dev::k_clear_first, 1, 1, 0, stream, st());
    check(cudaGetLastError(), "solve setup");
    // the iteration graph (recorded once per precision and smoother version)
    const int gi = refine ? 3 : (mixed ? 2 : (own16 ? 1 : 0));
    pend.graph = gi;
    if (graph[gi] && graphVersion[gi] != M->version) {
        cudaGraphExecDestroy(graph[gi]);
        graph[gi] = nullptr;
    }
    if (!graph[gi]) {
        cudaGraph_t gr;
        // the kernels of one replay: the launches made while recording (the fold branch's are
        // counted per fold; a graph's node types are not queried, the driver does not report the
        // conditional node's)
        const int64_t l0 = launches;
        check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "capture");
        if (mixed) recordMixedIteration(ctl, refine, half);
        else recordPlainIteration(ctl, own16);
        check(cudaStreamEndCapture(stream, &gr), "capture end");
        graphKernels[gi] = launches - l0;
        launches = l0;  // captured, not run
        check(cudaGraphInstantiate(&graph[gi], gr, 0), "instantiate");
        cudaGraphDestroy(gr);
        graphVersion[gi] = M->version;
    }
    enqueueStateRead();
}

bool SolverImpl::advance(bool block, ps_solve_result& res) {
    if (!pend.active) return true;
    if (block) check(cudaEventSynchronize(ev), "sync");
    else {
        const cudaError_t qe = cudaEventQuery(ev);
        if (qe == cudaErrorNotReady) return false;
        check(qe, "event query");
    }
    if (pend.lanczos) {
        pend.lanczos = false;
        if (lzPending) finishLanczos();
        computeCoefficients();
        startIterations();
        return false;
    }
    const HostLevel& h = H.levels[0];
    DevLevel& D = L[0];
    const int64_t n = pd(0);
    const ps_solve_opts& o = pend.o;
    const bool mixed = pend.mixed;
    const dev::Ctl none{nullptr, nullptr};
    if (!pend.finishing) {
        const dev::SolveState& hs = *hostState;
        bool stop = hs.done != 0;
        if (!stop && o.cancel && *o.cancel) {
            pend.outcome = PS_CANCELLED;
            stop = true;
        }
        if (!stop && o.time_limit_s > 0 &&
            std::chrono::duration<double>(std::chrono::steady_clock::now() - pend.t0).count() > o.time_limit_s) {
            pend.outcome = PS_TIMEOUT;
            stop = true;
        }
        if (!stop) {
            // the next batch of iterations, sized from the observed convergence rate
            const double rel = mixed ? std::max(hs.est, 0.0) : hs.rel;
            if (pend.lastIt > 0 && hs.it > pend.lastIt && rel > 0 && pend.lastRel > 0) {
                const double rate = std::pow(rel / pend.lastRel, 1.0 / (hs.it - pend.lastIt));
                int need = 32;
                if (rate < 0.999) need = int(std::ceil(std::log(o.tol / rel) / std::log(rate)));
                pend.batch = std::max(1, std::min({need, 32, 2 * pend.batch}));
            }
            pend.lastRel = rel;
            pend.lastIt = hs.it;
            const int batch = std::max(1, std::min(pend.batch, o.max_iter - hs.it + 1));
            const int gi = pend.graph;
            for (int b = 0; b < batch; b++) check(cudaGraphLaunch(graph[gi], stream), "graph launch");
            launches += int64_t(batch) * graphKernels[gi];
            enqueueStateRead();
            return false;
        }
        // the result: true residual, u to its destinations
        if (hs.done == 2) check(cudaMemsetAsync(x.p, 0, size_t(n) * 8, stream), "memset");
        if (!mixed) {
            op64(0, x.as<double>(), q.as<double>(), false, none);
            launch(dev::k_final, vecGrid(pn(0)), dev::VEC_THREADS, 0, stream, pn(0), D.view.nmask, f.as<double>(), q.as<double>(), st(), part(),
                   tick());
        } else if (pend.outcome == PS_CANCELLED || pend.outcome == PS_TIMEOUT) {
            // fold what the FP32 iterate holds and report the true residual
            launch(dev::k_mx_fold1, vecGrid(n), dev::VEC_THREADS, 0, stream, n, x.as<double>(), x32.as<float>(), st(), none);
            op64(0, x.as<double>(), q.as<double>(), false, none);
            launch(dev::k_final, vecGrid(pn(0)), dev::VEC_THREADS, 0, stream, pn(0), D.view.nmask, f.as<double>(), q.as<double>(), st(), part(),
                   tick());
        }
        // u to the caller in the dense layout (q is free here: the staging vector of the download)
        if (pend.uDev) pitch(x.as<double>(), pend.uDev, 0, false);
        if (pend.uHost) downloadPitched(x.as<double>(), pend.uHost, 0, q.as<double>());
        enqueueStateRead();
        pend.finishing = true;
        return false;
    }
    check(cudaGetLastError(), "solve");
    const dev::SolveState& hs = *hostState;
    if (hs.err) {
        pend.active = false;
        throw Error(PS_ECUDA, hs.err == dev::ST_ERR_STAGING ? "a tiled operator kernel gave up waiting for its staged data"
                                                            : "a tiled operator kernel found its shared memory misaligned");
    }
    ps_status outcome = pend.outcome;
    res.iterations = hs.it;
    res.residual = hs.rel;
    res.folds = hs.folds;
    res.converged = (outcome == PS_OK) && std::isfinite(hs.rel) && hs.rel <= o.tol * 10;
    if (outcome == PS_OK) {
        if (hs.status == dev::ST_BREAKDOWN && !res.converged) outcome = PS_BREAKDOWN;
        else if (!res.converged) outcome = PS_NOT_CONVERGED;
    }
    res.status = outcome;
    res.kernels = launches - pend.launches0 + (pend.mixed ? int64_t(hs.folds) * foldKernels : 0);
    res.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - pend.t0).count();
    pend.active = false;
    return true;
}

// ==================================================================== block (multi-RHS) solves
//
// Up to RB right-hand sides of one model solved together (the sizing study's load groups,
// native/src/fea/study_runner.cpp:453-465, and LOBPCG's block preconditioning, native/src/fea/
// eigen.cpp:508-513): every kernel of the iteration takes the whole block, so voxel words, masks and
// Galerkin matrices are read once per block instead of once per right-hand side. Each right-hand
// side keeps its own flexible CG (FP64 Krylov, FP32 V-cycle as in the single solve).

struct BlockBase {
    virtual ~BlockBase() = default;
    virtual int width() const = 0;
    virtual int64_t deviceBytes() const = 0;
    virtual int64_t launchCount() const = 0;
    // nrhs <= width() solves; f and u: nrhs consecutive dense vectors (host when host, else device);
    // x0 (same place as f) or null
    virtual ps_status solve(int nrhs, const double* f, const double* x0, bool host, const ps_solve_opts& o, double* u,
                            ps_solve_result* res) = 0;
    // z = one V-cycle applied to each of nvec <= width() dense device vectors r (voxel_fea.cpp:830-861)
    virtual void precondition(int nvec, const double* rDev, double* zDev, cudaStream_t caller) = 0;
};

template <int RB>
struct BlockImpl final : BlockBase {
    std::shared_ptr<SharedModel> M;
    Hierarchy& H;
    std::vector<DevLevel>& L;
    int smCount;
    std::vector<LevelWork> W;     // FP32 V-cycle vectors per level, RB wide
    DevMem f, x, r, p, q, z64;    // FP64 vectors of the finest level, RB wide
    DevMem state, partials, ticket;
    dev::BlockState* hostState = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev = nullptr;
    int64_t bytes = 0, launches = 0;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int64_t graphKernels[2] = {0, 0};
    int64_t graphVersion[2] = {-1, -1};

    BlockImpl(std::shared_ptr<SharedModel> model) : M(std::move(model)), H(M->H), L(M->L), smCount(M->smCount) {
        M->ensureActiveLists();
        M->ensureBlockStencils();
        static std::once_flag attrOnce;
        std::call_once(attrOnce, [] {
            // the stencil rows a CTA's warps stage (31 KB for an 8-wide block)
            auto set = [](auto kernel, size_t b) {
                check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(b)), "attr");
            };
            set(dev::kb_op<float, dev::BOP_CHEB, false, RB, true>, dev::stnBlockSmem<float>(32 / RB));
            set(dev::kb_op<float, dev::BOP_RESID, false, RB, true>, dev::stnBlockSmem<float>(32 / RB));
        });
        check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream");
        check(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "event");
        check(cudaMallocHost(&hostState, sizeof(dev::BlockState)), "cudaMallocHost");
        W.resize(L.size());
        for (size_t l = 0; l < W.size(); l++) {
            const size_t n = size_t(pd(int(l))) * RB * 4;
            W[l].r.alloc(n, bytes, stream);
            W[l].z.alloc(n, bytes, stream);
            W[l].t.alloc(n, bytes, stream);
            W[l].d.alloc(n, bytes, stream);
        }
        const size_t n = size_t(pd(0)) * RB * 8;
        for (DevMem* b : {&f, &x, &r, &p, &q}) b->alloc(n, bytes, stream);
        if (M->exactOneLevel()) z64.alloc(n, bytes, stream);
        state.alloc(sizeof(dev::BlockState), bytes, stream);
        partials.alloc(size_t(smCount) * 16 * RB * 3 * sizeof(double) + 4096, bytes, stream);
        ticket.alloc(64, bytes, stream);
        check(cudaStreamWaitEvent(stream, M->readyEv, 0), "wait");
    }
    ~BlockImpl() override {
        cudaStreamSynchronize(stream);
        for (auto& g : graph)
            if (g) cudaGraphExecDestroy(g);
        for (auto& w : W) w.release();
        for (DevMem* b : {&f, &x, &r, &p, &q, &z64, &state, &partials, &ticket}) b->release();
        if (ev) cudaEventDestroy(ev);
        if (hostState) cudaFreeHost(hostState);
        cudaStreamSynchronize(stream);
        cudaStreamDestroy(stream);
    }

    static int64_t bytesFor(const Hierarchy& H) {
        int64_t b = 0;
        for (const HostLevel& h : H.levels) b += 16 * int64_t(3) * pitch4(h.NX) * h.NY * h.NZ * RB;
        const HostLevel& h0 = H.levels[0];
        b += 6 * 8 * int64_t(3) * pitch4(h0.NX) * h0.NY * h0.NZ * RB;
        return b;
    }

    int width() const override { return RB; }
    int64_t deviceBytes() const override { return bytes; }
    int64_t launchCount() const override { return launches; }

    template <class... KArgs, class... Args>
    void launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, Args&&... args) {
        kernel<<<grid, block, smem, stream>>>(std::forward<Args>(args)...);
        ++launches;
    }
    int64_t pn(int l) const { return L[size_t(l)].view.nNodes; }
    int64_t pd(int l) const { return 3 * pn(l); }
    const int* act(int l) const { return M->act[size_t(l)].template as<int>(); }
    int nAct(int l) const { return M->nAct[size_t(l)]; }
    // grid of a kernel with one lane per (active node, right-hand side)
    int laneGrid(int l) const { return gridFor(int64_t(nAct(l)) * RB, dev::BLOCK_THREADS, smCount * 8); }
    int elemGrid(int l) const { return gridFor(int64_t(nAct(l)) * 3 * RB, dev::BLOCK_THREADS, smCount * 8); }
    dev::BlockState* bs() const { return state.as<dev::BlockState>(); }
    double* part() const { return partials.as<double>(); }
    unsigned* tick() const { return ticket.as<unsigned>(); }

    template <class T, int MODE>
    void op(int l, const T* xin, T* y, float c1, float c2, bool raw, bool own16, dev::Ctl ctl) {
        DevLevel& D = L[size_t(l)];
        if (!nAct(l)) return;
        float* rr = W[size_t(l)].r.template as<float>();
        float* dd = W[size_t(l)].d.template as<float>();
        if constexpr (sizeof(T) == 4 && RB == 32 && MODE != dev::BOP_DOT) {
            if (own16 && l == 0 && M->blockTc && M->nBtTiles > 0) {
                // the mixed form's finest level on the tensor cores (TF32)
                launch(dev::kb_tc<MODE>, M->nBtTiles, dev::BT_THREADS, dev::btSmemBytes(), D.view, static_cast<const dev::Coefs<float>&>(D.c32),
                       M->btTiles.template as<uint32_t>(), xin, y, rr, dd, c1, c2, raw ? 1 : 0, ctl);
                return;
            }
        }
        const auto& C = [&]() -> const dev::Coefs<T>& {
            if constexpr (sizeof(T) == 8) return D.c64;
            else return D.c32;
        }();
        // the assembled stencils of the Galerkin levels
        if constexpr (sizeof(T) == 4) {
            const float* stn = M->bstn32.empty() ? nullptr : M->bstn32[size_t(l)].template as<float>();
            if (stn) {
                launch(dev::kb_op<float, MODE, false, RB, true>, laneGrid(l), dev::BLOCK_THREADS, dev::stnBlockSmem<float>(32 / RB), D.view, C,
                       act(l), nAct(l), stn, xin, y, rr, dd, c1, c2, raw ? 1 : 0, bs(), part(), tick(), ctl);
                return;
            }
        }
        if (own16 && D.hasOwn)
            launch(dev::kb_op<T, MODE, true, RB>, laneGrid(l), dev::BLOCK_THREADS, 0, D.view, C, act(l), nAct(l), static_cast<const T*>(nullptr),
                   xin, y, rr, dd, c1, c2, raw ? 1 : 0, bs(), part(), tick(), ctl);
        else
            launch(dev::kb_op<T, MODE, false, RB>, laneGrid(l), dev::BLOCK_THREADS, 0, D.view, C, act(l), nAct(l), static_cast<const T*>(nullptr),
                   xin, y, rr, dd, c1, c2, raw ? 1 : 0, bs(), part(), tick(), ctl);
    }

    void coarse(const float* rin, float* zout, dev::Ctl ctl) {
        const int warpsNeeded = (M->m + (32 / RB) - 1) / (32 / RB);
        const int grid = std::max(1, std::min(smCount * 8, (warpsNeeded + 7) / 8));
        launch(dev::kb_coarse<float, float, RB>, grid, dev::BLOCK_THREADS, 0, M->m, M->cDof.template as<int>(), M->cInv.template as<double>(),
               rin, zout, ctl);
    }

    // the block V-cycle on level l from W[l].r (voxel_fea.cpp:817-828); returns the result buffer
    float* vcycle(int l, dev::Ctl ctl, bool own16, bool firstDone) {
        DevLevel& D = L[size_t(l)];
        LevelWork& Wl = W[size_t(l)];
        float *z = Wl.z.template as<float>(), *t = Wl.t.template as<float>(), *rl = Wl.r.template as<float>(), *d = Wl.d.template as<float>();
        const int last = int(L.size()) - 1;
        if (l == last) {
            if (H.hasFactor()) {
                coarse(rl, z, ctl);
                return z;
            }
            if (!firstDone)
                launch(dev::kb_cheb_first<RB>, elemGrid(l), dev::BLOCK_THREADS, 0, act(l), nAct(l), D.invD.template as<float>(), rl, d, z, D.omega,
                       ctl);
            float* a = z;
            float* b = t;
            for (int s = 1; s < 40; s++) {
                op<float, dev::BOP_CHEB>(l, a, b, 0.f, D.omega, false, own16, ctl);
                std::swap(a, b);
            }
            return a;
        }
        DevLevel& C = L[size_t(l + 1)];
        LevelWork& Wc = W[size_t(l + 1)];
        if (!firstDone)
            launch(dev::kb_cheb_first<RB>, elemGrid(l), dev::BLOCK_THREADS, 0, act(l), nAct(l), D.invD.template as<float>(), rl, d, z, D.cf0, ctl);
        float* a = z;
        float* b = t;
        for (size_t k = 0; k < D.chebC1.size(); k++) {
            op<float, dev::BOP_CHEB>(l, a, b, D.chebC1[k], D.chebC2[k], false, own16, ctl);
            std::swap(a, b);
        }
        op<float, dev::BOP_RESID>(l, a, b, 0.f, 0.f, false, own16, ctl);
        const bool fuse = !(l + 1 == last && H.hasFactor());
        const float c0c = (l + 1 == last) ? C.omega : C.cf0;
        launch(dev::kb_restrict<RB>, laneGrid(l + 1), dev::BLOCK_THREADS, 0, D.view, C.view, act(l + 1), nAct(l + 1), b, Wc.r.template as<float>(),
               fuse ? Wc.d.template as<float>() : nullptr, fuse ? Wc.z.template as<float>() : nullptr, c0c, ctl);
        float* zc = vcycle(l + 1, ctl, own16, fuse);
        launch(dev::kb_prolong<RB>, laneGrid(l), dev::BLOCK_THREADS, 0, D.view, C.view.PX, C.view.NY, act(l), nAct(l), zc, a, ctl);
        op<float, dev::BOP_CHEB>(l, a, b, 0.f, D.cf0, false, own16, ctl);
        std::swap(a, b);
        for (size_t k = 0; k < D.chebC1.size(); k++) {
            op<float, dev::BOP_CHEB>(l, a, b, D.chebC1[k], D.chebC2[k], false, own16, ctl);
            std::swap(a, b);
        }
        return a;
    }

    // z of the finest level: the V-cycle (from the fused first step) or the direct solve
    const float* precond(dev::Ctl ctl, bool own16) {
        if (M->exactOneLevel()) {
            const int warpsNeeded = (M->m + (32 / RB) - 1) / (32 / RB);
            const int grid = std::max(1, std::min(smCount * 8, (warpsNeeded + 7) / 8));
            launch(dev::kb_coarse<double, double, RB>, grid, dev::BLOCK_THREADS, 0, M->m, M->cDof.template as<int>(),
                   M->cInv.template as<double>(), r.template as<double>(), z64.template as<double>(), ctl);
            return nullptr;
        }
        return vcycle(0, ctl, own16, true);
    }

    void recordIteration(dev::Ctl ctl, bool own16) {
        DevLevel& D = L[0];
        LevelWork& W0 = W[0];
        op<double, dev::BOP_DOT>(0, p.template as<double>(), q.template as<double>(), 0.f, 0.f, false, false, ctl);
        const bool one = M->exactOneLevel();
        launch(dev::kb_cg_update<RB>, laneGrid(0), dev::BLOCK_THREADS, 0, act(0), nAct(0), D.view.nmask, x.template as<double>(),
               r.template as<double>(), p.template as<double>(), q.template as<double>(), W0.r.template as<float>(), D.invD.template as<float>(),
               W0.d.template as<float>(), W0.z.template as<float>(), one ? 0.f : D.cf0, bs(), part(), tick(), ctl);
        const float* z32 = precond(ctl, own16);
        launch(dev::kb_cg_dots<RB>, laneGrid(0), dev::BLOCK_THREADS, 0, act(0), nAct(0), D.view.nmask, r.template as<double>(), z32,
               one ? z64.template as<double>() : nullptr, q.template as<double>(), bs(), part(), tick(), ctl);
        launch(dev::kb_cg_p<RB>, laneGrid(0), dev::BLOCK_THREADS, 0, act(0), nAct(0), D.view.nmask, z32, one ? z64.template as<double>() : nullptr,
               p.template as<double>(), bs(), ctl);
    }

    // dense <-> block (device to device); scale per right-hand side or null
    void pack(const double* dense, int nrhs, double* blk, bool toBlock, const double* scale = nullptr) {
        const dev::LevelView& v = L[0].view;
        const int64_t nDense = int64_t(3) * v.NX * v.NY * v.NZ;
        launch(dev::kb_pack<RB>, gridFor(nDense, 32, smCount * 16), 256, 0, const_cast<double*>(dense), nrhs, (long long)nDense, blk, v.NX,
               v.NY, v.PX, toBlock ? 1 : 0, scale);
    }

    void readState() {
        check(cudaMemcpyAsync(hostState, state.p, sizeof(dev::BlockState), cudaMemcpyDeviceToHost, stream), "state read");
        check(cudaEventRecord(ev, stream), "event");
        check(cudaEventSynchronize(ev), "sync");
    }

    ps_status solve(int nrhs, const double* fIn, const double* x0In, bool host, const ps_solve_opts& o, double* uOut,
                    ps_solve_result* res) override {
        const auto t0 = std::chrono::steady_clock::now();
        const int64_t launches0 = launches;
        DevLevel& D = L[0];
        LevelWork& W0 = W[0];
        const HostLevel& h0 = H.levels[0];
        const size_t nDense = size_t(h0.nDof);
        const bool own16 = o.precision == PS_PREC_MIXED && M->mixedOwn16;
        const dev::Ctl none{nullptr, nullptr};
        const dev::Ctl ctl{&bs()->allDone, nullptr};
        // inputs: q holds the dense staging (RB >= nrhs vectors fit in one block vector)
        double* stage = q.template as<double>();
        auto bring = [&](const double* src, double* dst) {
            if (host) {
                check(cudaMemcpyAsync(stage, src, nDense * nrhs * 8, cudaMemcpyHostToDevice, stream), "upload");
                pack(stage, nrhs, dst, true);
            } else {
                pack(src, nrhs, dst, true);
            }
        };
        check(cudaMemsetAsync(x.p, 0, x.bytes, stream), "memset");
        check(cudaMemsetAsync(p.p, 0, p.bytes, stream), "memset");
        bring(fIn, f.template as<double>());
        if (x0In) {
            bring(x0In, x.template as<double>());
            launch(dev::kb_mask_fixed<RB>, gridFor(pn(0) * 3 * RB, dev::BLOCK_THREADS, smCount * 8), dev::BLOCK_THREADS, 0, pn(0), D.view.nmask,
                   x.template as<double>());
        }
        dev::BlockState s{};
        s.tol = o.tol;
        s.maxIter = o.max_iter;
        s.first = 1;
        s.nrhs = nrhs;
        *hostState = s;
        check(cudaMemcpyAsync(state.p, hostState, sizeof s, cudaMemcpyHostToDevice, stream), "state");
        op<double, dev::BOP_APPLY>(0, x.template as<double>(), q.template as<double>(), 0.f, 0.f, false, false, none);
        launch(dev::kb_cg_init<RB>, laneGrid(0), dev::BLOCK_THREADS, 0, act(0), nAct(0), D.view.nmask, f.template as<double>(),
               q.template as<double>(), r.template as<double>(), bs(), part(), tick());
        const bool one = M->exactOneLevel();
        launch(dev::kb_vc_load<RB>, laneGrid(0), dev::BLOCK_THREADS, 0, act(0), nAct(0), D.view.nmask, r.template as<double>(),
               W0.r.template as<float>(), D.invD.template as<float>(), W0.d.template as<float>(), W0.z.template as<float>(), one ? 0.f : D.cf0,
               bs(), ctl);
        const float* z32 = precond(ctl, own16);
        launch(dev::kb_cg_dots<RB>, laneGrid(0), dev::BLOCK_THREADS, 0, act(0), nAct(0), D.view.nmask, r.template as<double>(), z32,
               one ? z64.template as<double>() : nullptr, q.template as<double>(), bs(), part(), tick(), ctl);
        launch(dev::kb_cg_p<RB>, laneGrid(0), dev::BLOCK_THREADS, 0, act(0), nAct(0), D.view.nmask, z32, one ? z64.template as<double>() : nullptr,
               p.template as<double>(), bs(), ctl);
        launch(dev::kb_clear_first, 1, 1, 0, bs());
        check(cudaGetLastError(), "block solve setup");
        const int gi = own16 ? 1 : 0;
        if (graph[gi] && graphVersion[gi] != M->version) {
            cudaGraphExecDestroy(graph[gi]);
            graph[gi] = nullptr;
        }
        if (!graph[gi]) {
            cudaGraph_t gr;
            const int64_t l0 = launches;
            check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "capture");
            recordIteration(ctl, own16);
            check(cudaStreamEndCapture(stream, &gr), "capture end");
            graphKernels[gi] = launches - l0;
            launches = l0;
            check(cudaGraphInstantiate(&graph[gi], gr, 0), "instantiate");
            cudaGraphDestroy(gr);
            graphVersion[gi] = M->version;
        }
        readState();
        ps_status outcome = PS_OK;
        int batch = 2, lastIt = 0;
        double lastRel = 0;
        while (!hostState->allDone) {
            if (o.cancel && *o.cancel) {
                outcome = PS_CANCELLED;
                break;
            }
            if (o.time_limit_s > 0 && std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > o.time_limit_s) {
                outcome = PS_TIMEOUT;
                break;
            }
            // the next batch of iterations, sized from the slowest right-hand side's convergence
            double rel = 0;
            for (int k = 0; k < nrhs; k++)
                if (!hostState->done[k]) rel = std::max(rel, hostState->rel[k]);
            const int it = hostState->iter;
            if (lastIt > 0 && it > lastIt && rel > 0 && lastRel > 0) {
                const double rate = std::pow(rel / lastRel, 1.0 / (it - lastIt));
                int need = 32;
                if (rate < 0.999) need = int(std::ceil(std::log(o.tol / rel) / std::log(rate)));
                batch = std::max(1, std::min({need, 32, 2 * batch}));
            }
            lastRel = rel;
            lastIt = it;
            const int nb = std::max(1, std::min(batch, o.max_iter - it + 1));
            for (int b = 0; b < nb; b++) check(cudaGraphLaunch(graph[gi], stream), "graph launch");
            launches += int64_t(nb) * graphKernels[gi];
            readState();
        }
        // zero loads: u = 0 (x holds 0 there unless a warm start was given)
        dev::BlockState fin = *hostState;
        for (int k = 0; k < nrhs; k++)
            if (fin.done[k] == 2) launch(dev::kb_zero_rhs<RB>, gridFor(pn(0) * 3, dev::BLOCK_THREADS, smCount * 8), dev::BLOCK_THREADS, 0, pn(0),
                                         x.template as<double>(), k);
        op<double, dev::BOP_APPLY>(0, x.template as<double>(), q.template as<double>(), 0.f, 0.f, false, false, none);
        launch(dev::kb_final<RB>, laneGrid(0), dev::BLOCK_THREADS, 0, act(0), nAct(0), D.view.nmask, f.template as<double>(),
               q.template as<double>(), bs(), part(), tick());
        if (host) {
            pack(stage, nrhs, x.template as<double>(), false);
            check(cudaMemcpyAsync(uOut, stage, nDense * nrhs * 8, cudaMemcpyDeviceToHost, stream), "download");
        } else {
            pack(uOut, nrhs, x.template as<double>(), false);
        }
        readState();
        check(cudaGetLastError(), "block solve");
        const dev::BlockState& hs = *hostState;
        ps_status worst = PS_OK;
        const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        for (int k = 0; k < nrhs; k++) {
            ps_solve_result rr{};
            rr.iterations = hs.it[k];
            rr.residual = hs.rel[k];
            rr.converged = outcome == PS_OK && std::isfinite(hs.rel[k]) && hs.rel[k] <= o.tol * 10;
            ps_status st = outcome;
            if (st == PS_OK) {
                if (hs.status[k] == dev::ST_BREAKDOWN && !rr.converged) st = PS_BREAKDOWN;
                else if (!rr.converged) st = PS_NOT_CONVERGED;
            }
            rr.status = st;
            rr.seconds = secs;
            rr.kernels = (launches - launches0);
            if (res) res[k] = rr;
            if (st > worst) worst = st;
        }
        return worst;
    }

    void precondition(int nvec, const double* rDev, double* zDev, cudaStream_t caller) override {
        DevLevel& D = L[0];
        LevelWork& W0 = W[0];
        const dev::Ctl none{nullptr, nullptr};
        if (caller && caller != stream) {
            check(cudaEventRecord(ev, caller), "event");
            check(cudaStreamWaitEvent(stream, ev, 0), "wait");
        }
        dev::BlockState s{};
        s.nrhs = nvec;
        *hostState = s;
        check(cudaMemcpyAsync(state.p, hostState, sizeof s, cudaMemcpyHostToDevice, stream), "state");
        check(cudaMemsetAsync(r.p, 0, r.bytes, stream), "memset");
        pack(rDev, nvec, r.template as<double>(), true);
        launch(dev::kb_rmax<RB>, laneGrid(0), dev::BLOCK_THREADS, 0, act(0), nAct(0), D.view.nmask, r.template as<double>(), bs(), part(), tick());
        check(cudaMemsetAsync(q.p, 0, q.bytes, stream), "memset");
        if (z64.p) check(cudaMemsetAsync(z64.p, 0, z64.bytes, stream), "memset");
        if (M->exactOneLevel()) {
            // the whole model is the coarsest level: its direct FP64 solve (voxel_fea.cpp:838-842)
            precond(none, false);
            pack(zDev, nvec, z64.template as<double>(), false);
        } else {
            launch(dev::kb_vc_load<RB>, laneGrid(0), dev::BLOCK_THREADS, 0, act(0), nAct(0), D.view.nmask, r.template as<double>(),
                   W0.r.template as<float>(), D.invD.template as<float>(), W0.d.template as<float>(), W0.z.template as<float>(), D.cf0, bs(),
                   none);
            const float* z32 = vcycle(0, none, false, true);
            launch(dev::kb_vc_store<RB>, elemGrid(0), dev::BLOCK_THREADS, 0, act(0), nAct(0), z32, q.template as<double>(), bs());
            pack(zDev, nvec, q.template as<double>(), false);
        }
        check(cudaGetLastError(), "block precondition");
        if (caller && caller != stream) {
            check(cudaEventRecord(ev, stream), "event");
            check(cudaStreamWaitEvent(caller, ev, 0), "wait");
        }
    }
};

// ==================================================================== Solver

struct SolverHandle {
    std::shared_ptr<SharedModel> model;
    std::unique_ptr<SolverImpl> main;
    std::vector<std::unique_ptr<SolverImpl>> extra;  // batch contexts, created on demand
    std::unique_ptr<BlockBase> block;                // the multi-RHS block context, created on demand
};

namespace {

// the block width for nrhs right-hand sides: the narrowest of 8, 16, 32 that holds them (or 32),
// narrowed while its vectors do not fit the free device memory (less 1 GB); 0 if none fits
int chooseBlockWidth(const Hierarchy& H, int nrhs) {
    size_t freeB = 0, totalB = 0;
    check(cudaMemGetInfo(&freeB, &totalB), "cudaMemGetInfo");
    const int64_t avail = int64_t(freeB) - (int64_t(1) << 30);
    int want = nrhs <= 8 ? 8 : (nrhs <= 16 ? 16 : 32);
    for (; want >= 8; want /= 2) {
        const int64_t need = want == 32 ? BlockImpl<32>::bytesFor(H) : (want == 16 ? BlockImpl<16>::bytesFor(H) : BlockImpl<8>::bytesFor(H));
        if (need <= avail) return want;
    }
    return 0;
}

std::unique_ptr<BlockBase> makeBlock(std::shared_ptr<SharedModel> M, int width) {
    if (width == 32) return std::make_unique<BlockImpl<32>>(std::move(M));
    if (width == 16) return std::make_unique<BlockImpl<16>>(std::move(M));
    return std::make_unique<BlockImpl<8>>(std::move(M));
}

}  // namespace

BlockBase* Solver::blockFor(int nrhs) {
    SolverHandle& Hd = *handle_;
    const int fits = Hd.block ? Hd.block->width() : 0;
    const int want = nrhs <= 8 ? 8 : (nrhs <= 16 ? 16 : 32);
    if (Hd.block && fits >= std::min(want, 32)) return Hd.block.get();
    Hd.block.reset();  // its memory first
    check(cudaStreamSynchronize(impl_->stream), "sync");
    const int w = chooseBlockWidth(impl_->H, nrhs);
    if (!w) return nullptr;
    impl_->prepareSmoothers();
    Hd.block = makeBlock(impl_->M, w);
    return Hd.block.get();
}

Solver::Solver(const int32_t dims[3], const float* density, double nu, const uint8_t* bc, int64_t coarsestMaxDof, const double* diagAdd) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        throw Error(PS_ENODEV, "no CUDA device is available");
    }
    auto model = std::make_shared<SharedModel>();
    model->build(dims, density, nu, bc, coarsestMaxDof, diagAdd);
    auto* I = new SolverImpl(model);
    impl_.reset(I);
    I->allocate();
    handle_.reset(new SolverHandle{model, nullptr, {}});
}

Solver::Solver(Hierarchy&& hier) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        throw Error(PS_ENODEV, "no CUDA device is available");
    }
    auto model = std::make_shared<SharedModel>();
    model->adopt(std::move(hier));
    auto* I = new SolverImpl(model);
    impl_.reset(I);
    I->allocate();
    handle_.reset(new SolverHandle{model, nullptr, {}});
}

int64_t estimateDeviceBytes(const Hierarchy& H) {
    // what SharedModel::adopt and one SolverImpl::allocate take, plus allocation slack
    int64_t b = 0, allocs = 0;
    for (size_t l = 0; l < H.levels.size(); l++) {
        const HostLevel& h = H.levels[l];
        // pitched sizes: rows of PX = NX rounded up to 4 nodes, px = nx rounded up to 4 words
        const int64_t nodes = int64_t(pitch4(h.NX)) * h.NY * h.NZ, dofs = 3 * nodes;
        b += 4 * int64_t(pitch4(h.nx)) * h.ny * h.nz + nodes + 6 * 576 * h.nOwn + 4 * dofs + (h.diagAdd.empty() ? 0 : 12 * dofs) +
             4 * (h.nNodes / 1024 + 1);
        if (l == 0) b += dofs;
        b += 16 * dofs;  // V-cycle vectors r, z, t, d
        allocs += 12;
    }
    const int64_t n = 3 * int64_t(pitch4(H.levels[0].NX)) * H.levels[0].NY * H.levels[0].NZ;
    b += 40 * n + 12 * n + (H.levels.size() == 1 ? 8 * n : 0);
    b += 4 * H.coarseM + 8 * H.coarseM * H.coarseM;
    b += 4096 * 32 + 64 * 1024;
    allocs += 16;
    return b + allocs * (64 << 10);
}

Solver::~Solver() {
    handle_.reset();
    impl_.reset();
}

const Hierarchy& Solver::hierarchy() const { return impl_->H; }
int64_t Solver::nDof() const { return impl_->H.levels[0].nDof; }
int64_t Solver::deviceBytes() const {
    int64_t b = impl_->M->bytes + impl_->bytes;
    for (auto& c : handle_->extra) b += c->bytes;
    if (handle_->block) b += handle_->block->deviceBytes();
    return b;
}
int64_t Solver::contextBytes() const { return impl_->bytes; }
double Solver::levelLmax(int l) const { return impl_->H.levels[size_t(l)].lmax; }

static void validateF(const double* f, const double* x0, int64_t n) {
    bool bad = false;
    parallelFor(n, [&](int64_t lo, int64_t hi) {
        for (int64_t i = lo; i < hi; i++)
            if (!std::isfinite(f[i]) || (x0 && !std::isfinite(x0[i]))) {
                bad = true;
                return;
            }
    }, 1 << 20);
    if (bad) throw Error(PS_ENONFINITE, "Forces and displacements must be finite numbers.");
}

ps_status Solver::solve(const double* f, const ps_solve_opts& o, double* u, ps_solve_result& res) {
    SolverImpl& I = *impl_;
    const int64_t n = nDof();
    validateF(f, o.x0, n);
    const auto t0 = std::chrono::steady_clock::now();
    I.uploadPitched(f, I.f.as<double>(), 0, I.q.as<double>());
    const double* x0 = nullptr;
    if (o.x0) {
        I.uploadPitched(o.x0, I.p.as<double>(), 0, I.q.as<double>());
        x0 = I.p.as<double>();
    }
    I.startSolve(I.f.as<double>(), x0, o, nullptr, u);
    while (!I.advance(true, res)) {
    }
    res.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return ps_status(res.status);
}

ps_status Solver::solveDevice(const double* fDev, const ps_solve_opts& o, double* uDev, ps_solve_result& res) {
    SolverImpl& I = *impl_;
    const double* x0 = o.x0;
    if (x0) {
        I.pitch(x0, I.p.as<double>(), 0, true);
        x0 = I.p.as<double>();
    }
    return I.runSolve(fDev, x0, o, uDev, res);
}

void Solver::begin(const double* fHost, const ps_solve_opts& o, double* uHost) {
    SolverImpl& I = *impl_;
    I.uploadPitched(fHost, I.f.as<double>(), 0, I.q.as<double>());
    const double* x0 = nullptr;
    if (o.x0) {
        I.uploadPitched(o.x0, I.p.as<double>(), 0, I.q.as<double>());
        x0 = I.p.as<double>();
    }
    I.startSolve(I.f.as<double>(), x0, o, nullptr, uHost);
}

bool Solver::poll(ps_solve_result& res) { return impl_->advance(false, res); }

ps_status Solver::solveBatch(int32_t nrhs, const double* f, const ps_solve_opts& base, double* u, ps_solve_result* results, int concurrency) {
    const int64_t n = nDof();
    validateF(f, nullptr, n * nrhs);
    if (base.x0) validateF(base.x0, nullptr, n * nrhs);
    const char* mode = std::getenv("PSFEA_BATCH_MODE");
    const bool contexts = mode && std::string(mode) == "contexts";
    if (base.precision != PS_PREC_FP32 && nrhs >= 2 && !contexts) {
        impl_->setDegree(base.smoother_degree > 0 ? base.smoother_degree : impl_->M->defaultDegree);
        if (BlockBase* B = blockFor(nrhs)) {
            ps_status worst = PS_OK;
            for (int c = 0; c < nrhs; c += B->width()) {
                const int k = std::min(B->width(), nrhs - c);
                ps_solve_opts o = base;
                o.x0 = nullptr;
                const ps_status st = B->solve(k, f + int64_t(c) * n, base.x0 ? base.x0 + int64_t(c) * n : nullptr, true, o, u + int64_t(c) * n,
                                              results ? results + c : nullptr);
                if (st > worst) worst = st;
            }
            return worst;
        }
    }
    // contexts: the handle's own plus extra ones, as many as free memory allows
    size_t freeB = 0, totalB = 0;
    check(cudaMemGetInfo(&freeB, &totalB), "cudaMemGetInfo");
    const int64_t per = impl_->bytes + (64 << 20);
    const int fit = int(std::max<int64_t>(0, (int64_t(freeB) - (int64_t(1) << 30)) / per));
    const int K = std::max(1, std::min({concurrency, int(nrhs), 1 + fit}));
    SolverHandle& Hd = *handle_;
    while (int(Hd.extra.size()) < K - 1) {
        auto c = std::make_unique<SolverImpl>(impl_->M);
        c->allocate();
        Hd.extra.push_back(std::move(c));
    }
    std::vector<SolverImpl*> ctx{impl_.get()};
    for (int k = 0; k + 1 < K; k++) ctx.push_back(Hd.extra[size_t(k)].get());
    std::vector<int> job(size_t(K), -1);
    int next = 0, left = nrhs;
    ps_status worst = PS_OK;
    auto startOn = [&](int k, int q) {
        SolverImpl& I = *ctx[size_t(k)];
        ps_solve_opts o = base;
        I.uploadPitched(f + int64_t(q) * n, I.f.as<double>(), 0, I.q.as<double>());
        const double* x0 = nullptr;
        if (base.x0) {
            I.uploadPitched(base.x0 + int64_t(q) * n, I.p.as<double>(), 0, I.q.as<double>());
            x0 = I.p.as<double>();
        }
        o.x0 = nullptr;
        I.startSolve(I.f.as<double>(), x0, o, nullptr, u + int64_t(q) * n);
        job[size_t(k)] = q;
    };
    // the smoothers are estimated once, before the contexts run side by side
    impl_->setDegree(base.smoother_degree > 0 ? base.smoother_degree : impl_->M->defaultDegree);
    impl_->prepareSmoothers();
    for (int k = 0; k < K && next < nrhs; k++) startOn(k, next++);
    while (left > 0) {
        bool progressed = false;
        for (int k = 0; k < K; k++) {
            if (job[size_t(k)] < 0) continue;
            ps_solve_result r{};
            if (!ctx[size_t(k)]->advance(false, r)) continue;
            progressed = true;
            const int q = job[size_t(k)];
            if (results) results[q] = r;
            if (r.status > worst) worst = ps_status(r.status);
            left--;
            job[size_t(k)] = -1;
            if (next < nrhs) startOn(k, next++);
        }
        if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
    return worst;
}

void Solver::precondition(const double* rHost, double* zHost) {
    SolverImpl& I = *impl_;
    const HostLevel& h = I.H.levels[0];
    DevLevel& D = I.L[0];
    LevelWork& W0 = I.W[0];
    const int64_t n = I.pd(0), nn = I.pn(0);
    I.setDegree(2);  // the reference's preconditioner
    I.prepareSmoothers();
    I.uploadPitched(rHost, I.r.as<double>(), 0, I.q.as<double>());
    const dev::Ctl none{nullptr, nullptr};
    if (I.exactOneLevel()) {
        // the whole model is the coarsest level: its direct FP64 solve (voxel_fea.cpp:838-842)
        const int threads = 256, warps = threads / 32;
        const int grid = std::max(1, std::min(I.smCount * 2, (I.m + warps - 1) / warps));
        check(cudaMemsetAsync(I.z64.p, 0, size_t(n) * 8, I.stream), "memset");
        I.launch(dev::k_coarse<double, double>, grid, threads, size_t(I.m) * sizeof(double), I.stream, I.m, I.cDof.as<int>(), I.cInv.as<double>(),
                 I.r.as<double>(), I.z64.as<double>(), 1.0, none);
        I.downloadPitched(I.z64.as<double>(), zHost, 0, I.q.as<double>());
    } else {
        I.launch(dev::k_rmax, I.vecGrid(nn), dev::VEC_THREADS, 0, I.stream, nn, D.view.nmask, I.r.as<double>(), I.st(), I.part(), I.tick());
        I.launch(dev::k_vc_load, I.vecGrid(nn), dev::VEC_THREADS, 0, I.stream, nn, D.view.nmask, I.r.as<double>(), W0.r.as<float>(),
                 D.invD.as<float>(), W0.d.as<float>(), W0.z.as<float>(), D.cf0, I.st(), none);
        float* z32 = I.vcycle(0, none, false, true);
        I.launch(dev::k_vc_store, I.vecGrid(nn), dev::VEC_THREADS, 0, I.stream, nn, D.view.nmask, z32, I.q.as<double>(), I.st());
        I.downloadPitched(I.q.as<double>(), zHost, 0, I.p.as<double>());
    }
    check(cudaStreamSynchronize(I.stream), "precondition");
}

void Solver::preconditionBlock(int32_t nvec, const double* rDev, double* zDev, void* s) {
    impl_->setDegree(2);  // the reference's preconditioner
    BlockBase* B = blockFor(nvec);
    if (!B) throw Error(PS_EOOM, "the block vectors do not fit the free device memory");
    const int64_t n = nDof();
    cudaStream_t caller = s ? static_cast<cudaStream_t>(s) : impl_->stream;
    for (int c = 0; c < nvec; c += B->width()) {
        const int k = std::min(B->width(), nvec - c);
        B->precondition(k, rDev + int64_t(c) * n, zDev + int64_t(c) * n, caller);
    }
}

void Solver::setStream(void* s) {
    SolverImpl& I = *impl_;
    cudaStream_t want = s ? static_cast<cudaStream_t>(s) : I.ownStream;
    if (want != I.stream) {
        // graphs were captured from the old stream's work; replays may go to any stream, so keep them
        check(cudaStreamSynchronize(I.stream), "sync");
        I.stream = want;
    }
}

double Solver::timeKernel(int which, int reps) {
    SolverImpl& I = *impl_;
    I.prepareSmoothers();
    const dev::Ctl none{nullptr, nullptr};
    DevLevel& D = I.L[0];
    LevelWork& W0 = I.W[0];
    cudaEvent_t e0, e1;
    check(cudaEventCreate(&e0), "event");
    check(cudaEventCreate(&e1), "event");
    auto once = [&] {
        if (which == 0) I.op32<dev::OP_CHEB>(0, W0.z.as<float>(), W0.t.as<float>(), D.cf1, D.cf2, none, true);
        else I.op64(0, I.p.as<double>(), I.q.as<double>(), false, none);
    };
    once();
    check(cudaEventRecord(e0, I.stream), "event");
    for (int k = 0; k < reps; k++) once();
    check(cudaEventRecord(e1, I.stream), "event");
    check(cudaEventSynchronize(e1), "event");
    float ms = 0;
    check(cudaEventElapsedTime(&ms, e0, e1), "event");
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return double(ms) / reps;
}

int64_t Solver::launches() const {
    int64_t n = impl_->launches;
    for (auto& c : handle_->extra) n += c->launches;
    if (handle_->block) n += handle_->block->launchCount();
    return n;
}

namespace {

// FNV-1a over the model's level-0 voxel words and node masks, its size, nu and level count: equal
// signatures mean the same operator, masks and hierarchy depth
uint64_t modelSignature(const Hierarchy& H) {
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](const void* p, size_t n) {
        const unsigned char* b = static_cast<const unsigned char*>(p);
        for (size_t i = 0; i < n; i++) {
            h ^= b[i];
            h *= 1099511628211ull;
        }
    };
    const HostLevel& L0 = H.levels[0];
    const int d[3] = {L0.nx, L0.ny, L0.nz};
    mix(d, sizeof d);
    mix(&H.nu, sizeof H.nu);
    const size_t nl = H.levels.size();
    mix(&nl, sizeof nl);
    mix(L0.word.data(), L0.word.size() * 4);
    mix(L0.nmask.data(), L0.nmask.size());
    return h;
}

std::mutex tuneMu;
std::map<uint64_t, TuneResult>& tuneCache() {
    static std::map<uint64_t, TuneResult> c;
    return c;
}

}  // namespace

TuneResult Solver::autotune(const double* fHost, const ps_solve_opts& base, bool force) {
    SolverImpl& I = *impl_;
    SharedModel& M = *I.M;
    const uint64_t sig = modelSignature(I.H);
    auto apply = [&](const TuneResult& t) {
        M.defaultDegree = t.degree;
        for (size_t l = 0; l < M.L.size(); l++) {
            DevLevel& D = M.L[l];
            if (!D.useTiles) continue;
            D.split32 = (t.splitLevels >> l) & 1;
            if (l == 0) D.inner64 = t.inner64 != 0;
        }
        M.version++;  // the iteration graphs are recorded again
    };
    if (!force) {
        std::lock_guard<std::mutex> g(tuneMu);
        auto it = tuneCache().find(sig);
        if (it != tuneCache().end()) {
            TuneResult t = it->second;
            apply(t);
            t.trials = 0;
            t.cached = 1;
            return t;
        }
    }
    const int64_t n = nDof();
    validateF(fHost, nullptr, n);
    int64_t scratch = 0;
    DevMem fDev, uDev;
    fDev.alloc(size_t(n) * 8, scratch);
    uDev.alloc(size_t(n) * 8, scratch);
    check(cudaMemcpy(fDev.p, fHost, size_t(n) * 8, cudaMemcpyHostToDevice), "upload");
    TuneResult cur;
    cur.degree = M.defaultDegree;
    for (size_t l = 0; l < M.L.size(); l++)
        if (M.L[l].useTiles && M.L[l].split32) cur.splitLevels |= int64_t(1) << l;
    cur.inner64 = (!M.L.empty() && M.L[0].inner64) ? 1 : 0;
    int trials = 0;
    auto timeOf = [&](const TuneResult& t) {
        apply(t);
        ps_solve_opts o = base;
        o.smoother_degree = t.degree;
        o.x0 = nullptr;
        ps_solve_result r{};
        I.runSolve(fDev.as<double>(), nullptr, o, uDev.as<double>(), r);  // records the graph, estimates smoothers
        const auto t0 = std::chrono::steady_clock::now();
        I.runSolve(fDev.as<double>(), nullptr, o, uDev.as<double>(), r);
        const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        trials++;
        return r.converged ? sec : 1e300;
    };
    const double t0 = timeOf(cur);
    TuneResult best = cur;
    double bestT = t0;
    for (int deg = 1; deg <= 4; deg++) {
        if (deg == cur.degree) continue;
        TuneResult t = best;
        t.degree = deg;
        const double s = timeOf(t);
        if (s < bestT) {
            bestT = s;
            best = t;
        }
    }
    // each tiled level's 32-bit split, then the finest level's 64-bit in-tile boundary nodes
    for (size_t l = 0; l < M.L.size(); l++) {
        if (!M.L[l].useTiles || !M.L[l].nBnd) continue;
        TuneResult t = best;
        t.splitLevels ^= int64_t(1) << l;
        const double s = timeOf(t);
        if (s < bestT) {
            bestT = s;
            best = t;
        }
    }
    if (!M.L.empty() && M.L[0].useTiles && M.L[0].nBnd) {
        TuneResult t = best;
        t.inner64 ^= 1;
        const double s = timeOf(t);
        if (s < bestT) {
            bestT = s;
            best = t;
        }
    }
    apply(best);
    best.trials = trials;
    best.bestSeconds = bestT;
    best.defaultSeconds = t0;
    best.cached = 0;
    {
        std::lock_guard<std::mutex> g(tuneMu);
        tuneCache()[sig] = best;
    }
    return best;
}

void Solver::apply(int level, const double* xHost, double* yHost, bool raw) {
    SolverImpl& I = *impl_;
    if (level < 0 || level >= int(I.L.size())) throw Error(PS_EINVAL, "level out of range");
    const int64_t n = I.pd(level);
    // p and q as level `level` vectors: cleared first, so their padding entries hold 0
    check(cudaMemsetAsync(I.p.p, 0, size_t(n) * 8, I.stream), "memset");
    I.uploadPitched(xHost, I.p.as<double>(), level, I.q.as<double>());
    check(cudaMemsetAsync(I.q.p, 0, size_t(n) * 8, I.stream), "memset");  // inactive tiles are not written
    I.op64(level, I.p.as<double>(), I.q.as<double>(), raw, dev::Ctl{nullptr, nullptr});
    I.downloadPitched(I.q.as<double>(), yHost, level, I.p.as<double>());
    check(cudaStreamSynchronize(I.stream), "apply");
}

void Solver::stresses(const double* u, double E, double h, bool principals, float* vm, float* p1, float* p3) {
    SolverImpl& I = *impl_;
    const HostLevel& L0 = I.H.levels[0];
    const int64_t nn = I.pn(0);
    const dev::LevelView& v = I.L[0].view;
    dev::StressCoefs sc;
    for (int a = 0; a < 8; a++)
        for (int i = 0; i < 144; i++) sc.S[a][i] = I.H.el.cornerStress[a][i] * E / h;
    int64_t scratch = 0;
    DevMem out;
    out.alloc(size_t(nn) * 4 * 6, scratch);  // three pitched fields and three dense ones
    I.uploadPitched(u, I.p.as<double>(), 0, I.q.as<double>());
    float* o = out.as<float>();
    I.launch(dev::k_stresses, I.nodeGrid(nn), dev::NODE_THREADS, 0, I.stream, v, sc, I.p.as<double>(), principals ? 1 : 0, o, o + nn,
             o + 2 * nn);
    const int64_t nd = L0.nNodes;
    float* outs[3] = {vm, p1, p3};
    for (int f = 0; f < (principals ? 3 : 1); f++) {
        float* dense = o + 3 * nn + f * nn;
        I.launch(dev::k_pitch<float>, I.vecGrid(nd), dev::VEC_THREADS, 0, I.stream, o + f * nn, dense, 1, v.NX, v.NY, v.NZ, v.PX, 0);
        check(cudaMemcpyAsync(outs[f], dense, size_t(nd) * 4, cudaMemcpyDeviceToHost, I.stream), "stress download");
    }
    check(cudaStreamSynchronize(I.stream), "stresses");
}

void Solver::reactions(const double* u, const double* f, double R[3]) {
    SolverImpl& I = *impl_;
    const HostLevel& L0 = I.H.levels[0];
    const int64_t n = I.pd(0);
    (void)L0;
    check(cudaMemsetAsync(I.p.p, 0, size_t(n) * 8, I.stream), "memset");
    I.uploadPitched(u, I.p.as<double>(), 0, I.q.as<double>());
    if (f) {
        check(cudaMemsetAsync(I.r.p, 0, size_t(n) * 8, I.stream), "memset");
        I.uploadPitched(f, I.r.as<double>(), 0, I.q.as<double>());
    }
    check(cudaMemsetAsync(I.q.p, 0, size_t(n) * 8, I.stream), "memset");
    I.op64(0, I.p.as<double>(), I.q.as<double>(), true, dev::Ctl{nullptr, nullptr});
    I.launch(dev::k_reactions, I.vecGrid(I.pn(0)), dev::VEC_THREADS, 0, I.stream, I.pn(0), I.L[0].view.nmask, I.L[0].bc.as<uint8_t>(),
             I.q.as<double>(), f ? I.r.as<double>() : nullptr, I.st(), I.part(), I.tick());
    I.readState();
    R[0] = I.hostState->alpha;
    R[1] = I.hostState->beta;
    R[2] = I.hostState->pq;
}

// ==================================================================== allocation-free product
//
// For callers that must not allocate device memory during a call: code running on device memory
// owned by another allocator (a framework's caching pool, a fixed serving budget) and loops that
// cannot afford the implicit device synchronisation a cudaMalloc may cause. y = K x and x.y on the
// finest level with the reduction's scratch (per-block partial sums and the last-block ticket) in
// this file-scope device array instead of handle-owned or newly allocated memory. Its size caps the
// kernel's grid at NOALLOC_BLOCKS blocks (grid-stride, so any model size fits); a device whose
// launch shape would need more is refused. Every call on a device shares the array: calls that
// overlap on the GPU race, and each call clears the ticket before use.

constexpr int NOALLOC_BLOCKS = 4096;
constexpr size_t NOALLOC_BYTES = 256 + size_t(NOALLOC_BLOCKS) * sizeof(double);  // ticket line + partials
static __device__ __align__(256) unsigned char g_noallocScratch[NOALLOC_BYTES];

namespace dev {

// q = K p (FP64, held DOFs 0) and p.q into *dot, the reduction scratch in g_noallocScratch
__global__ void __launch_bounds__(NODE_THREADS) k_apply_dot_static(LevelView L, Coefs<double> C, const double* __restrict__ p,
                                                                   double* __restrict__ q, double* __restrict__ dot,
                                                                   unsigned char* scratch) {
    // p and q are the caller's vectors in the reference's dense layout (node nd = i + NX (j + NY k));
    // masks, words and the diagonal shift are the level's pitched arrays
    double v[1] = {0.0};
    const long long nDense = (long long)L.NX * L.NY * L.NZ;
    for (long long nd = blockIdx.x * (long long)blockDim.x + threadIdx.x; nd < nDense; nd += (long long)gridDim.x * blockDim.x) {
        const long long row = nd / L.NX;
        const int i = int(nd - row * L.NX), j = int(row % L.NY), k = int(row / L.NY);
        const long long n = i + (long long)L.PX * row;
        const uint8_t mask = __ldg(L.nmask + n);
        double acc[3];
        applyAt<double, false>(L, C, p, i, j, k, nd, mask, acc, L.NX, n);
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const double y = fixedDof(mask, c) ? 0.0 : acc[c];
            q[3 * nd + c] = y;
            v[0] += p[3 * nd + c] * y;
        }
    }
    unsigned* ticket = reinterpret_cast<unsigned*>(scratch);
    double* partials = reinterpret_cast<double*>(scratch + 256);
    double tot[1];
    if (gridReduce<1>(v, 0u, partials, ticket, tot) && threadIdx.x == 0) *dot = tot[0];
}

}  // namespace dev

namespace {

// device address of g_noallocScratch on device devId (the current device), looked up once per
// device (the first call on a device does it, so that first call should come before any stream
// capture)
unsigned char* noallocScratch(int devId) {
    static std::mutex mu;
    static std::vector<unsigned char*> addr;
    std::lock_guard<std::mutex> lock(mu);
    if (int(addr.size()) <= devId) addr.resize(size_t(devId) + 1, nullptr);
    if (!addr[size_t(devId)]) {
        void* p = nullptr;
        check(cudaGetSymbolAddress(&p, g_noallocScratch), "cudaGetSymbolAddress");
        addr[size_t(devId)] = static_cast<unsigned char*>(p);
    }
    return addr[size_t(devId)];
}

}  // namespace

void Solver::applyDotStatic(const double* xDev, double* yDev, double* dotDev, void* s) {
    SolverImpl& I = *impl_;
    const HostLevel& h = I.H.levels[0];
    DevLevel& D = I.L[0];
    const int grid = I.nodeGrid(h.nNodes);
    if (grid > NOALLOC_BLOCKS)
        throw Error(PS_EINVAL, "this device needs " + std::to_string(grid) + " reduction blocks; the static scratch holds " +
                                   std::to_string(NOALLOC_BLOCKS));
    int cur = -1;
    check(cudaGetDevice(&cur), "cudaGetDevice");
    if (cur != I.M->devId)
        throw Error(PS_EINVAL, "the current CUDA device is " + std::to_string(cur) + "; the handle lives on device " +
                                   std::to_string(I.M->devId));
    cudaStream_t st = s ? static_cast<cudaStream_t>(s) : I.stream;
    // a caller's stream is ordered after the model's uploads (the handle's own stream already is)
    if (st != I.stream) check(cudaStreamWaitEvent(st, I.M->readyEv, 0), "wait for the model");
    unsigned char* scratch = noallocScratch(cur);
    check(cudaMemsetAsync(scratch, 0, 256, st), "ticket clear");
    I.launch(dev::k_apply_dot_static, grid, dev::NODE_THREADS, 0, st, D.view, D.c64, xDev, yDev, dotDev, scratch);
    check(cudaGetLastError(), "apply_dot_static");
}

}  // namespace psfea
