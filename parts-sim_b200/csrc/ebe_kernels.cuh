// Element-block operator on the tensor cores (sm_100a tcgen05). Included by solver.cu only.
//
// On a level whose voxels are all s * Kb (the finest level: no Galerkin matrices), y = K x is
// sum over voxels of s_v Kb u_v scattered to the voxel's 8 corners. One CTA owns an 8 x 8 x 4 tile
// of nodes; the solid voxels of its 9 x 9 x 5 footprint are compacted (increasing voxel index) into
// the rows of A = [u_v - u_v,corner0] (rows x 24, the corner-0 value subtracted per component: Kb
// annihilates translations, so the product is unchanged and the TF32 rounding scales with the
// local variation), and one elected thread multiplies A by Kb^T (24 x 24, padded to N = 32) with
// tcgen05.mma kind::tf32 into tensor memory, 128 rows per instruction group. With SPLIT = 3 the
// product is the three-term split hi*hi + hi*lo + lo*hi (hi = the TF32 truncation, lo = the rest),
// close to FP32 accuracy. The rows come back with tcgen05.ld, scaled by s_v, into shared memory,
// and every owned node sums its up-to-8 voxel rows in a fixed order (deterministic), then runs the
// tile kernel's epilogue (APPLY / CHEB / RESID).
//
// Shared-memory operands use the canonical K-major layout without swizzle: element (row, k) of an
// R-row operand at byte (k / 8) (R / 8) 256 + ((k % 8) / 4) 128 + (row / 8) 256 + (row % 8) 16 +
// (k % 4) 4, i.e. 8-row x 16-byte core matrices, leading-dimension offset 128 B, stride-dimension
// offset 256 B, one 8-wide k-step per (R / 8) 256 B. Waits on the MMA completion barrier are
// bounded: a timeout records ST_ERR_STAGING and ends the solve; tensor memory is freed on every path.
#pragma once

#include "kernels.cuh"

namespace psfea {
namespace dev {

constexpr int EX = 8, EY = 8, EZ = 4, EBE_NODES = EX * EY * EZ, EBE_THREADS = 256;
constexpr int EVX = EX + 1, EVY = EY + 1, EVZ = EZ + 1, EBE_VOX = EVX * EVY * EVZ;    // 405 footprint voxels
constexpr int EHX = EX + 2, EHY = EY + 2, EHZ = EZ + 2, EBE_HALO = EHX * EHY * EHZ;  // 600 halo nodes
constexpr int EBE_GROUPS = (EBE_VOX + 127) / 128;                                    // 4 row groups of 128
constexpr int EBE_YSTRIDE = 25;                                                      // Y rows (bank spread)
constexpr uint32_t EBE_GROUP_BYTES = 128 * 24 * 4;                                   // one A group: 12288 B
constexpr uint32_t EBE_TMEM_COLS = 128;                                              // 4 groups x N 32
static_assert(EBE_VOX <= EBE_GROUPS * 128, "row groups");
static_assert(EBE_NODES == EBE_THREADS, "one owned node per thread");

__host__ __device__ constexpr uint32_t ebeCanon(int row, int k, int R) {
    return uint32_t((k / 8) * (R / 8) * 256 + ((k % 8) / 4) * 128 + (row / 8) * 256 + (row % 8) * 16 + (k % 4) * 4);
}
template <int SPLIT> __host__ __device__ constexpr uint32_t ebeBytesA() {
    const uint32_t a = uint32_t(SPLIT == 3 ? 2 : 1) * EBE_GROUPS * EBE_GROUP_BYTES, y = uint32_t(EBE_GROUPS) * 128 * EBE_YSTRIDE * 4;
    return a > y ? a : y;
}
template <int SPLIT> __host__ __device__ constexpr uint32_t ebeOffB() { return ebeBytesA<SPLIT>(); }
template <int SPLIT> __host__ __device__ constexpr uint32_t ebeOffX() { return ebeOffB<SPLIT>() + 2 * 32 * 24 * 4; }
template <int SPLIT> __host__ __device__ constexpr uint32_t ebeOffW() { return ebeOffX<SPLIT>() + align128(EBE_HALO * 3 * 4); }
template <int SPLIT> __host__ __device__ constexpr uint32_t ebeOffRow() { return ebeOffW<SPLIT>() + align128(EBE_VOX * 4); }
template <int SPLIT> __host__ __device__ constexpr uint32_t ebeOffVox() { return ebeOffRow<SPLIT>() + align128(EBE_VOX * 2); }
template <int SPLIT> __host__ __device__ constexpr uint32_t ebeOffMisc() { return ebeOffVox<SPLIT>() + align128(EBE_GROUPS * 128 * 2); }
template <int SPLIT> __host__ __device__ constexpr size_t ebeSmemBytes() { return ebeOffMisc<SPLIT>() + 128 + 1024; }  // + alignment slack

// UMMA shared-memory descriptor: start address, leading / stride byte offsets (16-byte units),
// descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t ummaDesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((addr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) | (uint64_t((sbo >> 4) & 0x3FFFu) << 32) |
           (uint64_t(1) << 46);
}
// instruction descriptor: FP32 accumulator, TF32 A and B, both K-major, N = 32, M = 128
constexpr uint32_t EBE_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void ummaTf32(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(EBE_IDESC), "r"(accumulate));
}
__device__ __forceinline__ float tf32Hi(float v) { return __uint_as_float(__float_as_uint(v) & 0xffffe000u); }

template <int MODE, int SPLIT>
__global__ void __launch_bounds__(EBE_THREADS, SPLIT == 3 ? 1 : 3)
    k_ebe(LevelView L, Coefs<float> C, const uint32_t* __restrict__ tiles, const float* __restrict__ x, float* __restrict__ y,
          const float* __restrict__ r, float* __restrict__ d, float c1, float c2, int raw, SolveState* st, Ctl ctl) {
    if (skipped(ctl)) return;
    extern __shared__ __align__(1024) unsigned char ebeRaw[];
    unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(ebeRaw) + 1023) & ~uintptr_t(1023));
    float* Ah = reinterpret_cast<float*>(sm);
    float* Al = reinterpret_cast<float*>(sm + EBE_GROUPS * EBE_GROUP_BYTES);
    float* Y = reinterpret_cast<float*>(sm);  // after the products: the scaled rows
    float* Bh = reinterpret_cast<float*>(sm + ebeOffB<SPLIT>());
    float* Bl = Bh + 32 * 24;
    float* xs = reinterpret_cast<float*>(sm + ebeOffX<SPLIT>());
    uint32_t* ws = reinterpret_cast<uint32_t*>(sm + ebeOffW<SPLIT>());
    int16_t* rowOf = reinterpret_cast<int16_t*>(sm + ebeOffRow<SPLIT>());
    int16_t* voxOf = reinterpret_cast<int16_t*>(sm + ebeOffVox<SPLIT>());
    int* scanW = reinterpret_cast<int*>(sm + ebeOffMisc<SPLIT>());  // 8 warp counts
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + ebeOffMisc<SPLIT>() + 64);
    uint32_t* tmemSlot = reinterpret_cast<uint32_t*>(sm + ebeOffMisc<SPLIT>() + 80);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t tw = tiles[blockIdx.x];
    const int i0 = int(tw & 2047u) * EX, j0 = int((tw >> 11) & 2047u) * EY, k0 = int(tw >> 22) * EZ;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smemAddr(tmemSlot)), "r"(EBE_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (tid == 0) mbarInit(bar, 1);
    // x halo (nodes i0-1 .. i0+EX, ...; outside the grid 0) and the footprint's voxel words
    for (int e = tid; e < EBE_HALO * 3; e += EBE_THREADS) {
        const int row = e / (EHX * 3), rem = e - row * EHX * 3, hx = rem / 3, c = rem - hx * 3;
        const int hy = row % EHY, hz = row / EHY;
        const int gi = i0 - 1 + hx, gj = j0 - 1 + hy, gk = k0 - 1 + hz;
        float v = 0.f;
        if (gi >= 0 && gj >= 0 && gk >= 0 && gi < L.NX && gj < L.NY && gk < L.NZ) v = __ldg(x + 3 * (gi + (long long)L.PX * (gj + (long long)L.NY * gk)) + c);
        xs[e] = v;
    }
    for (int e = tid; e < EBE_VOX; e += EBE_THREADS) {
        const int vx = e % EVX, vy = (e / EVX) % EVY, vz = e / (EVX * EVY);
        const int gi = i0 - 1 + vx, gj = j0 - 1 + vy, gk = k0 - 1 + vz;
        ws[e] = (gi >= 0 && gj >= 0 && gk >= 0 && gi < L.nx && gj < L.ny && gk < L.nz) ? __ldg(L.word + L.wi(gi, gj, gk)) : 0u;
    }
    // Kb^T as the B operand (rows 24-31 zero)
    for (int e = tid; e < 32 * 24; e += EBE_THREADS) {
        const int n = e / 24, k = e - n * 24;
        const float v = n < 24 ? C.Kb[n * 24 + k] : 0.f;
        const float hi = tf32Hi(v);
        Bh[ebeCanon(n, k, 32) / 4] = hi;
        if (SPLIT == 3) Bl[ebeCanon(n, k, 32) / 4] = v - hi;
    }
    __syncthreads();
    // solid voxels -> rows, in increasing voxel order
    int nRows = 0;
    for (int rnd = 0; rnd < (EBE_VOX + EBE_THREADS - 1) / EBE_THREADS; rnd++) {
        const int v = rnd * EBE_THREADS + tid;
        const bool f = v < EBE_VOX && ws[v] != 0;
        const unsigned bal = __ballot_sync(0xffffffffu, f);
        if (lane == 0) scanW[warp] = __popc(bal);
        __syncthreads();
        int pre = 0, total = 0;
#pragma unroll
        for (int k = 0; k < EBE_THREADS / 32; k++) {
            const int c = scanW[k];
            pre += k < warp ? c : 0;
            total += c;
        }
        if (v < EBE_VOX) {
            const int row = f ? nRows + pre + __popc(bal & ((1u << lane) - 1)) : -1;
            rowOf[v] = int16_t(row);
            if (f) voxOf[row] = int16_t(v);
        }
        nRows += total;
        __syncthreads();
    }
    // the A rows: each voxel's 24 corner values less its corner-0 value
    for (int row = tid; row < nRows; row += EBE_THREADS) {
        const int v = voxOf[row], vx = v % EVX, vy = (v / EVX) % EVY, vz = v / (EVX * EVY);
        float e[24];
#pragma unroll
        for (int b = 0; b < 8; b++) {
            const int bx = (b == 1 || b == 2 || b == 5 || b == 6), by = (b == 2 || b == 3 || b == 6 || b == 7), bz = b >> 2;
            const float* xp = xs + 3 * ((vx + bx) + EHX * ((vy + by) + EHY * (vz + bz)));
            e[3 * b] = xp[0];
            e[3 * b + 1] = xp[1];
            e[3 * b + 2] = xp[2];
        }
        const float b0 = e[0], b1 = e[1], b2 = e[2];
#pragma unroll
        for (int b = 0; b < 8; b++) {
            e[3 * b] -= b0;
            e[3 * b + 1] -= b1;
            e[3 * b + 2] -= b2;
        }
        const int g = row >> 7, rr = row & 127;
        unsigned char* ah = reinterpret_cast<unsigned char*>(Ah) + g * EBE_GROUP_BYTES;
        unsigned char* al = reinterpret_cast<unsigned char*>(Al) + g * EBE_GROUP_BYTES;
#pragma unroll
        for (int q = 0; q < 6; q++) {
            const float4 hi = make_float4(tf32Hi(e[4 * q]), tf32Hi(e[4 * q + 1]), tf32Hi(e[4 * q + 2]), tf32Hi(e[4 * q + 3]));
            *reinterpret_cast<float4*>(ah + ebeCanon(rr, 4 * q, 128)) = hi;
            if (SPLIT == 3)
                *reinterpret_cast<float4*>(al + ebeCanon(rr, 4 * q, 128)) =
                    make_float4(e[4 * q] - hi.x, e[4 * q + 1] - hi.y, e[4 * q + 2] - hi.z, e[4 * q + 3] - hi.w);
        }
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *tmemSlot;
    const int nGroups = (nRows + 127) >> 7;
    if (tid == 0 && nGroups > 0) {
        for (int g = 0; g < nGroups; g++)
#pragma unroll
            for (int kk = 0; kk < 3; kk++) {
                const uint64_t aH = ummaDesc(smemAddr(Ah) + g * EBE_GROUP_BYTES + kk * 4096, 128, 256);
                const uint64_t bH = ummaDesc(smemAddr(Bh) + kk * 1024, 128, 256);
                ummaTf32(tmem + 32 * g, aH, bH, kk > 0);
                if (SPLIT == 3) {
                    ummaTf32(tmem + 32 * g, aH, ummaDesc(smemAddr(Bl) + kk * 1024, 128, 256), 1);
                    ummaTf32(tmem + 32 * g, ummaDesc(smemAddr(Al) + g * EBE_GROUP_BYTES + kk * 4096, 128, 256), bH, 1);
                }
            }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smemAddr(bar)) : "memory");
    }
    const bool ok = nGroups == 0 || mbarWait(bar, TILE_WAIT_POLLS);
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (ok) {
        // rows back from tensor memory: warp w reads lanes 32 (w % 4) .. + 31 of groups w / 4, w / 4 + 2
        const int q4 = warp & 3;
        for (int g = warp >> 2; g < nGroups; g += 2) {
            uint32_t v[32];
            const uint32_t addr = tmem + uint32_t(32 * g) + (uint32_t(32 * q4) << 16);
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,%20,%21,%"
                "22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]),
                  "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]),
                  "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]),
                  "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                : "r"(addr));
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
            const int row = 128 * g + 32 * q4 + lane;
            if (row < nRows) {
                const float s = __uint_as_float(ws[voxOf[row]]);
#pragma unroll
                for (int n = 0; n < 24; n++) Y[row * EBE_YSTRIDE + n] = s * __uint_as_float(v[n]);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    const bool good = __syncthreads_and(ok) != 0;
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(EBE_TMEM_COLS) : "memory");
    if (!good) {
        if (tid == 0) {
            atomicExch(&st->err, ST_ERR_STAGING);
            st->done = 1;
        }
        return;
    }
    // the owned node of this thread: its voxels' rows in a fixed order, then the epilogue
    const int cx = tid % EX, cy = (tid / EX) % EY, cz = tid / (EX * EY);
    const int gi = i0 + cx, gj = j0 + cy, gk = k0 + cz;
    if (gi >= L.PX || gj >= L.NY || gk >= L.NZ) return;
    const long long n = gi + (long long)L.PX * (gj + (long long)L.NY * gk);
    const uint8_t mask = __ldg(L.nmask + n);
    const bool act = mask & NM_ACTIVE;
    float kx[3] = {0.f, 0.f, 0.f};
    if (act) {
#pragma unroll
        for (int vv = 0; vv < 8; vv++) {
            const int di = vv & 1, dj = (vv >> 1) & 1, dk = vv >> 2;
            const int row = rowOf[(cx + di) + EVX * ((cy + dj) + EVY * (cz + dk))];
            if (row < 0) continue;
            const int a = cornerOf(1 - di, 1 - dj, 1 - dk);
            const float* yr = Y + row * EBE_YSTRIDE + 3 * a;
            kx[0] += yr[0];
            kx[1] += yr[1];
            kx[2] += yr[2];
        }
    }
    const float* xo = xs + 3 * ((cx + 1) + EHX * ((cy + 1) + EHY * (cz + 1)));
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const long long id = 3 * n + c;
        const bool fx = fixedDof(mask, c);
        float k = act ? kx[c] : 0.f;
        if (act && L.dadd32) k += L.dadd32[id] * xo[c];
        if constexpr (MODE == TOP_APPLY) {
            y[id] = (!raw && fx) ? 0.f : k;
        } else if constexpr (MODE == TOP_RESID) {
            y[id] = fx ? 0.f : r[id] - k;
        } else {
            if (fx) {
                d[id] = 0.f;
                y[id] = 0.f;
            } else {
                const float dn = c1 * d[id] + c2 * __ldg(L.invD + id) * (r[id] - k);
                d[id] = dn;
                y[id] = xo[c] + dn;
            }
        }
    }
}

}  // namespace dev
}  // namespace psfea
