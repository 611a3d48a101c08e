// Study loops on the device: SIMP topology optimisation (native/src/fea/topology.cpp:103-183, with
// the solve of native/src/fea/study_runner.cpp:403-419) and the break test (native/src/fea/
// static_study.cpp:199-279). Each iteration's solve is the device solver warm-started from the
// previous displacements, which stay in device memory; the per-voxel work of the loops (density
// filter and its transpose, element energies, the optimality-criteria update and its volume
// bisection, the failure measure) runs as kernels next to it. The model of each iteration is
// rebuilt from the new densities (host hierarchy and Galerkin coarsening, then upload).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "element.hpp"
#include "host_util.hpp"
#include "hierarchy.hpp"
#include "solver.hpp"
#include "study.hpp"

namespace psfea {

namespace {

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error(PS_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

template <class T>
struct Dev {
    T* p = nullptr;
    size_t n = 0;
    Dev() = default;
    explicit Dev(size_t count) { alloc(count); }
    Dev(const Dev&) = delete;
    Dev& operator=(const Dev&) = delete;
    ~Dev() {
        if (p) cudaFree(p);
    }
    void alloc(size_t count) {
        if (p) cudaFree(p);
        p = nullptr;
        n = count;
        if (count) {
            ck(cudaMalloc(&p, count * sizeof(T)), "cudaMalloc");
            ck(cudaMemset(p, 0, count * sizeof(T)), "cudaMemset");
        }
    }
    void upload(const T* src, size_t count) { ck(cudaMemcpy(p, src, count * sizeof(T), cudaMemcpyHostToDevice), "upload"); }
    void download(T* dst, size_t count) const { ck(cudaMemcpy(dst, p, count * sizeof(T), cudaMemcpyDeviceToHost), "download"); }
};

constexpr int RT = 256;        // threads of the reduction kernels
constexpr int MAX_OFFS = 256;  // filter offsets (rmin up to ~3.5 voxels)

struct FilterOffsets {
    int n;
    int di[MAX_OFFS], dj[MAX_OFFS], dk[MAX_OFFS];
    double w[MAX_OFFS];
};

struct Mat24 {
    double K[576];
};

// ---- deterministic reductions: per-block sums (fixed tree), folded in block order by one block

__device__ __forceinline__ double blockSum(double v, bool isMax) {
    __shared__ double sh[RT];
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int o = RT / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] = isMax ? fmax(sh[threadIdx.x], sh[threadIdx.x + o]) : sh[threadIdx.x] + sh[threadIdx.x + o];
        __syncthreads();
    }
    return sh[0];
}

// partials[block] = sum over i of a[i] * (b ? b[i] : 1), or with free: a[q] * (free[q] ? b[q] : 1)
__global__ void k_sum(long long n, const double* __restrict__ a, const double* __restrict__ b, const uint8_t* __restrict__ isFree,
                      double* __restrict__ partials) {
    double s = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double bv = b ? ((isFree && !isFree[i]) ? 1.0 : b[i]) : 1.0;
        s += a[i] * bv;
    }
    const double t = blockSum(s, false);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
}

// partials[block] = max over i of |a[i] - b[i]|
__global__ void k_maxdiff(long long n, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ partials) {
    double s = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        s = fmax(s, fabs(a[i] - b[i]));
    const double t = blockSum(s, true);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
}

__global__ void k_fold(int nb, const double* __restrict__ partials, double* __restrict__ out, int isMax) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s = 0;
    for (int b = 0; b < nb; b++) s = isMax ? fmax(s, partials[b]) : s + partials[b];
    *out = s;
}

// ---- SIMP (topology.cpp)

// per design voxel q: the filter weight sum W[q] = sum of max(0, rmin - distance) over the design
// voxels in reach (topology.cpp:20-52)
__global__ void k_filter_w(int m, const int* __restrict__ ids, const int* __restrict__ pos, int nx, int ny, int nz, FilterOffsets F,
                           double* __restrict__ W) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < m; q += gridDim.x * blockDim.x) {
        const int e = ids[q], i = e % nx, j = (e / nx) % ny, k = e / (nx * ny);
        double s = 0;
        for (int t = 0; t < F.n; t++) {
            const int a = i + F.di[t], b = j + F.dj[t], c = k + F.dk[t];
            if (a < 0 || b < 0 || c < 0 || a >= nx || b >= ny || c >= nz) continue;
            if (pos[a + nx * (b + ny * c)] >= 0) s += F.w[t];
        }
        W[q] = s;
    }
}

// out = the density filter of x (topology.cpp:54-62); transpose: out[q] = sum w g[p] / W[p]
// (:66-77). keepOne: kept voxels (not free) read 1.
__global__ void k_filter(int m, const int* __restrict__ ids, const int* __restrict__ pos, int nx, int ny, int nz, FilterOffsets F,
                         const double* __restrict__ W, const double* __restrict__ x, double* __restrict__ out, int transpose,
                         const uint8_t* __restrict__ keepOne) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < m; q += gridDim.x * blockDim.x) {
        const int e = ids[q], i = e % nx, j = (e / nx) % ny, k = e / (nx * ny);
        double s = 0;
        for (int t = 0; t < F.n; t++) {
            const int a = i + F.di[t], b = j + F.dj[t], c = k + F.dk[t];
            if (a < 0 || b < 0 || c < 0 || a >= nx || b >= ny || c >= nz) continue;
            const int p = pos[a + nx * (b + ny * c)];
            if (p < 0) continue;
            s += transpose ? F.w[t] * x[p] / W[p] : F.w[t] * x[p];
        }
        double v = transpose ? s : s / W[q];
        if (keepOne && !keepOne[q]) v = 1.0;
        out[q] = v;
    }
}

// voxel densities of the solve: fill * (xmin + (1 - xmin) xPhys^p), at most 1 (topology.cpp:126-127)
__global__ void k_topo_density(int m, const int* __restrict__ ids, const double* __restrict__ fill, const double* __restrict__ xPhys, double penal,
                               double xmin, float* __restrict__ density) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < m; q += gridDim.x * blockDim.x)
        density[ids[q]] = float(fmin(1.0, fill[q] * (xmin + (1 - xmin) * pow(xPhys[q], penal))));
}

// u_e^T K0 u_e per design voxel (unit stiffness, no density scale; topology.cpp:79-100), and the
// compliance sensitivity dc = -p (1 - xmin) fill xPhys^(p-1) energy (:133-136)
__global__ void k_topo_sens(int m, const int* __restrict__ ids, int nx, int ny, const double* __restrict__ u, Mat24 K0,
                            const double* __restrict__ fill, const double* __restrict__ xPhys, double penal, double xmin, double* __restrict__ dc) {
    const long long NX = nx + 1, NY = ny + 1;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < m; q += gridDim.x * blockDim.x) {
        const int e = ids[q], i = e % nx, j = (e / nx) % ny, k = e / (nx * ny);
        const long long base = i + NX * (j + NY * k);
        const long long off[8] = {0, 1, 1 + NX, NX, NX * NY, 1 + NX * NY, 1 + NX + NX * NY, NX + NX * NY};
        double ue[24];
#pragma unroll
        for (int a = 0; a < 8; a++)
#pragma unroll
            for (int d = 0; d < 3; d++) ue[3 * a + d] = u[3 * (base + off[a]) + d];
        double s = 0;
        for (int r = 0; r < 24; r++) {
            double t = 0;
#pragma unroll
            for (int c = 0; c < 24; c++) t += K0.K[r * 24 + c] * ue[c];
            s += ue[r] * t;
        }
        dc[q] = -penal * (1 - xmin) * fill[q] * pow(xPhys[q], penal - 1) * s;
    }
}

// the optimality-criteria update for multiplier lm (topology.cpp:150-156)
__global__ void k_topo_oc(int m, const double* __restrict__ x, const double* __restrict__ dcx, const double* __restrict__ dvx,
                          const uint8_t* __restrict__ isFree, double lm, double move, double* __restrict__ xNew) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < m; q += gridDim.x * blockDim.x) {
        if (!isFree[q]) {
            xNew[q] = 1;
            continue;
        }
        const double B = sqrt(fmax(0.0, -dcx[q]) / (lm * dvx[q] + 1e-300));
        xNew[q] = fmax(0.0, fmax(x[q] - move, fmin(1.0, fmin(x[q] + move, x[q] * B))));
    }
}

__global__ void k_scatter_f(int m, const int* __restrict__ ids, const double* __restrict__ v, float* __restrict__ out) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < m; q += gridDim.x * blockDim.x) out[ids[q]] = float(v[q]);
}

// ---- break test (static_study.cpp:199-279)

// per solved voxel: the worst of its 8 corner nodal stresses (static_study.cpp:233-240)
__global__ void k_break_measure(long long nVox, int nx, int ny, const float* __restrict__ density, const float* __restrict__ nodal,
                                float* __restrict__ measure) {
    const long long NX = nx + 1, NY = ny + 1;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nVox; e += (long long)gridDim.x * blockDim.x) {
        float mv = 0.f;
        if (density[e] > 0) {
            const long long i = e % nx, j = (e / nx) % ny, k = e / ((long long)nx * ny);
            const long long base = i + NX * (j + NY * k);
            const long long off[8] = {0, 1, 1 + NX, NX, NX * NY, 1 + NX * NY, 1 + NX + NX * NY, NX + NX * NY};
#pragma unroll
            for (int a = 0; a < 8; a++) mv = fmaxf(mv, nodal[base + off[a]]);
        } else {
            mv = -1.f;  // not a solved voxel
        }
        measure[e] = mv;
    }
}

struct Reducer {
    int nb, smCount;
    Dev<double> partials, out;
    explicit Reducer(int sm) : nb(sm * 2), smCount(sm), partials(size_t(sm) * 2), out(1) {}
    double fold(bool isMax) {
        k_fold<<<1, 32>>>(nb, partials.p, out.p, isMax ? 1 : 0);
        double v = 0;
        out.download(&v, 1);
        return v;
    }
    double sum(long long n, const double* a, const double* b, const uint8_t* isFree = nullptr) {
        k_sum<<<nb, RT>>>(n, a, b, isFree, partials.p);
        return fold(false);
    }
    double maxdiff(long long n, const double* a, const double* b) {
        k_maxdiff<<<nb, RT>>>(n, a, b, partials.p);
        return fold(true);
    }
};

int gridOf(int64_t n, int sm) { return int(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, int64_t(sm) * 8))); }

int smCountNow() {
    int dev = 0, sm = 148;
    ck(cudaGetDevice(&dev), "cudaGetDevice");
    ck(cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev), "attribute");
    return sm;
}

// ---- pruneFloating on the device (voxel_fea.cpp:1086-1119): the voxels face-connected to a voxel
// touching a held node survive. The reference walks them breadth-first; here the solid voxels'
// 6-connected components are found by a lock-free union-find (roots hooked under the smaller index
// by compare-and-swap, paths halved on the way), and a voxel survives when its component holds a
// voxel with a held corner. The surviving set is unique, so the result equals the reference's.

constexpr int UF_MAX_STEPS = 1 << 24;  // bound on any find / hook loop (a bad state ends the kernel)

__device__ __forceinline__ int ufFind(int* p, int x, int* err) {
    for (int s = 0; s < UF_MAX_STEPS; s++) {
        const int px = p[x];
        if (px == x) return x;
        const int gp = p[px];
        if (gp != px) p[x] = gp;  // path halving; any value written is an ancestor, so it is safe
        x = gp;
    }
    atomicExch(err, 1);
    return x;
}

__global__ void k_uf_init(long long nVox, const float* __restrict__ density, int* __restrict__ parent) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nVox; e += (long long)gridDim.x * blockDim.x)
        parent[e] = density[e] > 0 ? int(e) : -1;
}

__global__ void k_uf_hook(long long nVox, int nx, int ny, int* __restrict__ parent, int* err) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nVox; e += (long long)gridDim.x * blockDim.x) {
        if (parent[e] < 0) continue;
        const long long i = e % nx, j = (e / nx) % ny;
        const long long nb[3] = {i + 1 < nx ? e + 1 : -1, j + 1 < ny ? e + nx : -1, e + (long long)nx * ny < nVox ? e + (long long)nx * ny : -1};
        for (int q = 0; q < 3; q++) {
            if (nb[q] < 0 || parent[nb[q]] < 0) continue;
            int a = int(e), b = int(nb[q]);
            for (int s = 0; s < UF_MAX_STEPS; s++) {
                a = ufFind(parent, a, err);
                b = ufFind(parent, b, err);
                if (a == b) break;
                if (a < b) {
                    const int t = a;
                    a = b;
                    b = t;
                }
                const int old = atomicCAS(parent + a, a, b);  // the larger root under the smaller
                if (old == a) break;
                a = old;
                if (s + 1 == UF_MAX_STEPS) atomicExch(err, 1);
            }
        }
    }
}

// roots of the components with a voxel touching a held node: flag[root] = 1
__global__ void k_uf_touch(long long nVox, int nx, int ny, const uint8_t* __restrict__ held, int* __restrict__ parent, int* __restrict__ flag,
                           int* err) {
    const long long NX = nx + 1, NY = ny + 1;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nVox; e += (long long)gridDim.x * blockDim.x) {
        if (parent[e] < 0) continue;
        const long long i = e % nx, j = (e / nx) % ny, k = e / ((long long)nx * ny);
        bool t = false;
#pragma unroll
        for (int a = 0; a < 8; a++) {
            const int bx = (a == 1 || a == 2 || a == 5 || a == 6), by = (a == 2 || a == 3 || a == 6 || a == 7), bz = a >> 2;
            t = t || held[(i + bx) + NX * ((j + by) + NY * (k + bz))] != 0;
        }
        if (t) flag[ufFind(parent, int(e), err)] = 1;
    }
}

__global__ void k_uf_keep(long long nVox, const float* __restrict__ density, int* __restrict__ parent, const int* __restrict__ flag,
                          float* __restrict__ out, int* __restrict__ removed, int* err) {
    int rem = 0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nVox; e += (long long)gridDim.x * blockDim.x) {
        float v = 0.f;
        if (parent[e] >= 0) {
            if (flag[ufFind(parent, int(e), err)]) v = density[e];
            else rem++;
        }
        out[e] = v;
    }
    if (rem) atomicAdd(removed, rem);
}

}  // namespace

int pruneFloatingDevice(const int32_t dims[3], const float* densityDev, const uint8_t* heldDev, float* outDev, void* streamPtr) {
    cudaStream_t stream = static_cast<cudaStream_t>(streamPtr);
    const int nx = dims[0], ny = dims[1], nz = dims[2];
    if (nx < 1 || ny < 1 || nz < 1) throw Error(PS_EINVAL, "The structural grid must have three positive dimensions.");
    const long long nVox = (long long)nx * ny * nz;
    if (nVox > (long long)INT32_MAX) throw Error(PS_EINVAL, "grid too large for 32-bit voxel labels");
    int* parent = nullptr;
    int* flag = nullptr;
    int* cnt = nullptr;  // removed, error
    ck(cudaMallocAsync(&parent, size_t(nVox) * 4, stream), "cudaMallocAsync");
    ck(cudaMallocAsync(&flag, size_t(nVox) * 4, stream), "cudaMallocAsync");
    ck(cudaMallocAsync(&cnt, 8, stream), "cudaMallocAsync");
    ck(cudaMemsetAsync(flag, 0, size_t(nVox) * 4, stream), "memset");
    ck(cudaMemsetAsync(cnt, 0, 8, stream), "memset");
    const int sm = smCountNow();
    const int g = gridOf(nVox, sm);
    k_uf_init<<<g, 256, 0, stream>>>(nVox, densityDev, parent);
    k_uf_hook<<<g, 256, 0, stream>>>(nVox, nx, ny, parent, cnt + 1);
    k_uf_touch<<<g, 256, 0, stream>>>(nVox, nx, ny, heldDev, parent, flag, cnt + 1);
    k_uf_keep<<<g, 256, 0, stream>>>(nVox, densityDev, parent, flag, outDev, cnt, cnt + 1);
    int h[2] = {0, 0};
    ck(cudaMemcpyAsync(h, cnt, 8, cudaMemcpyDeviceToHost, stream), "download");
    cudaFreeAsync(parent, stream);
    cudaFreeAsync(flag, stream);
    cudaFreeAsync(cnt, stream);
    ck(cudaStreamSynchronize(stream), "prune");
    if (h[1]) throw Error(PS_ECUDA, "the component labelling did not settle");
    return h[0];
}

bool deviceAvailable() {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return false;
    }
    return true;
}

int topologyRun(const int32_t dims[3], const float* fill, const uint8_t* keep, double nu, const uint8_t* bc, const double* f,
                const TopologyOptions& o, float* densityOut, std::vector<TopologyStep>& history) {
    const int nx = dims[0], ny = dims[1], nz = dims[2];
    if (nx < 1 || ny < 1 || nz < 1) throw Error(PS_EINVAL, "The structural grid must have three positive dimensions.");
    const int64_t nVox = int64_t(nx) * ny * nz, nDof = 3 * int64_t(nx + 1) * (ny + 1) * (nz + 1);
    if (nVox > int64_t(INT32_MAX)) throw Error(PS_EINVAL, "grid too large");
    const double xmin = 1e-3;  // TOPO_XMIN (topology.hpp:22)
    const int sm = smCountNow();
    // design voxels (fill > 0), their volumes and free flags (topology.cpp:104-118)
    std::vector<int> ids;
    for (int64_t e = 0; e < nVox; e++)
        if (fill[e] > 0) ids.push_back(int(e));
    const int m = int(ids.size());
    if (m == 0) throw Error(PS_EINVAL, "No voxels to optimise.");
    std::vector<double> vol(static_cast<size_t>(m));
    std::vector<uint8_t> isFree(size_t(m), 0);
    double totalVol = 0, keptVol = 0;
    for (int q = 0; q < m; q++) {
        vol[size_t(q)] = fill[ids[size_t(q)]];
        totalVol += vol[size_t(q)];
        if (keep && keep[ids[size_t(q)]]) keptVol += vol[size_t(q)];
        else isFree[size_t(q)] = 1;
    }
    const double target = std::max(o.volFrac * totalVol, keptVol * 1.02);
    const double start = std::min(1.0, std::max(xmin, (target - keptVol) / std::max(1e-12, totalVol - keptVol)));
    std::vector<double> x(static_cast<size_t>(m));
    for (int q = 0; q < m; q++) x[size_t(q)] = isFree[size_t(q)] ? start : 1;
    // filter offsets in the reference's order (k, j, i), weights rmin - distance > 0 (topology.cpp:22-31)
    FilterOffsets F{};
    {
        const int r = int(std::ceil(o.rmin)) - 1;
        for (int k = -r - 1; k <= r + 1; k++)
            for (int j = -r - 1; j <= r + 1; j++)
                for (int i = -r - 1; i <= r + 1; i++) {
                    const double w = o.rmin - std::sqrt(double(i * i + j * j + k * k));
                    if (!(w > 0)) continue;
                    if (F.n >= MAX_OFFS) throw Error(PS_EINVAL, "filter radius too large");
                    F.di[F.n] = i;
                    F.dj[F.n] = j;
                    F.dk[F.n] = k;
                    F.w[F.n] = w;
                    F.n++;
                }
    }
    std::vector<int> pos(size_t(nVox), -1);
    for (int q = 0; q < m; q++) pos[size_t(ids[size_t(q)])] = q;
    Mat24 K0;
    {
        const HexElement el = hexElement(nu);
        std::memcpy(K0.K, el.K, sizeof K0.K);
    }
    Dev<int> dIds(static_cast<size_t>(m)), dPos(static_cast<size_t>(nVox));
    Dev<double> dFill(static_cast<size_t>(m)), dW(static_cast<size_t>(m)), dX(static_cast<size_t>(m)), dXPhys(static_cast<size_t>(m)), dDc(static_cast<size_t>(m)), dDcx(static_cast<size_t>(m)), dDvx(static_cast<size_t>(m)),
        dXNew(static_cast<size_t>(m)), dPhys(static_cast<size_t>(m)), dVol(static_cast<size_t>(m)), dF(static_cast<size_t>(nDof)), dU(static_cast<size_t>(nDof));
    Dev<uint8_t> dFree(static_cast<size_t>(m));
    Dev<float> dDensity(static_cast<size_t>(nVox));
    dIds.upload(ids.data(), size_t(m));
    dPos.upload(pos.data(), size_t(nVox));
    dFill.upload(vol.data(), size_t(m));  // fill of each design voxel = its volume
    dVol.upload(vol.data(), size_t(m));
    dX.upload(x.data(), size_t(m));
    dFree.upload(isFree.data(), size_t(m));
    dF.upload(f, size_t(nDof));
    Reducer R(sm);
    const int g = gridOf(m, sm);
    k_filter_w<<<g, 256>>>(m, dIds.p, dPos.p, nx, ny, nz, F, dW.p);
    std::vector<float> density(size_t(nVox), 0.f);
    double change = 1;
    bool haveU = false;
    for (int it = 0; it < o.maxIter; it++) {
        const auto t0 = std::chrono::steady_clock::now();
        k_filter<<<g, 256>>>(m, dIds.p, dPos.p, nx, ny, nz, F, dW.p, dX.p, dXPhys.p, 0, dFree.p);
        k_topo_density<<<g, 256>>>(m, dIds.p, dFill.p, dXPhys.p, o.penal, xmin, dDensity.p);
        ck(cudaGetLastError(), "topology");
        dDensity.download(density.data(), size_t(nVox));
        // the iteration's model and its warm-started solve (study_runner.cpp:403-419)
        Solver S(dims, density.data(), nu, bc, 1100, nullptr);
        ps_solve_opts so;
        ps_solve_opts_default(&so);
        so.tol = o.solveTol;
        so.max_iter = 3000;
        so.precision = o.precision;
        so.x0 = haveU ? dU.p : nullptr;
        ps_solve_result sr{};
        const ps_status st = S.solveDevice(dF.p, so, dU.p, sr);
        ck(cudaDeviceSynchronize(), "topology solve");
        if (st == PS_CANCELLED || st == PS_TIMEOUT) throw Error(st, "the solve was stopped");
        haveU = true;
        k_topo_sens<<<g, 256>>>(m, dIds.p, nx, ny, dU.p, K0, dFill.p, dXPhys.p, o.penal, xmin, dDc.p);
        const double c = R.sum(nDof, dF.p, dU.p);
        const double used = R.sum(m, dVol.p, dXPhys.p);
        TopologyStep hs;
        hs.it = it;
        hs.compliance = c;
        hs.volume = used / totalVol;
        hs.change = change;
        hs.solveIterations = sr.iterations;
        hs.solveStatus = st;
        if (it > 4 && change < o.tol) {
            hs.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            history.push_back(hs);
            break;
        }
        k_filter<<<g, 256>>>(m, dIds.p, dPos.p, nx, ny, nz, F, dW.p, dDc.p, dDcx.p, 1, nullptr);
        k_filter<<<g, 256>>>(m, dIds.p, dPos.p, nx, ny, nz, F, dW.p, dVol.p, dDvx.p, 1, nullptr);
        // optimality criteria: bisection on the volume multiplier (topology.cpp:146-163)
        double l1 = 0, l2 = 1e9;
        while ((l2 - l1) / (l1 + l2 + 1e-30) > 1e-4) {
            const double lm = 0.5 * (l1 + l2);
            k_topo_oc<<<g, 256>>>(m, dX.p, dDcx.p, dDvx.p, dFree.p, lm, o.move, dXNew.p);
            k_filter<<<g, 256>>>(m, dIds.p, dPos.p, nx, ny, nz, F, dW.p, dXNew.p, dPhys.p, 0, nullptr);
            const double v = R.sum(m, dVol.p, dPhys.p, dFree.p);
            if (v > target) l1 = lm;
            else l2 = lm;
        }
        change = R.maxdiff(m, dXNew.p, dX.p);
        std::swap(dX.p, dXNew.p);
        hs.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        history.push_back(hs);
    }
    k_filter<<<g, 256>>>(m, dIds.p, dPos.p, nx, ny, nz, F, dW.p, dX.p, dXPhys.p, 0, dFree.p);
    ck(cudaMemset(dDensity.p, 0, size_t(nVox) * 4), "memset");
    k_scatter_f<<<g, 256>>>(m, dIds.p, dXPhys.p, dDensity.p);
    ck(cudaGetLastError(), "topology");
    dDensity.download(densityOut, size_t(nVox));
    return int(history.size());
}

BreakReason breakTest(const int32_t dims[3], const float* density0, double nu, const uint8_t* bc, const double* f, double E, double h,
                      double strength, bool principal, int maxSteps, std::vector<BreakStep>& steps, float* densityOut, double& peak) {
    if (!(strength > 0)) throw Error(PS_EINVAL, "Failure strength must be positive.");
    const int nx = dims[0], ny = dims[1], nz = dims[2];
    if (nx < 1 || ny < 1 || nz < 1) throw Error(PS_EINVAL, "The structural grid must have three positive dimensions.");
    const int64_t nVox = int64_t(nx) * ny * nz, NX = nx + 1, NY = ny + 1, nNodes = NX * NY * (nz + 1), nDof = 3 * nNodes;
    const int sm = smCountNow();
    std::vector<uint8_t> held(size_t(nNodes), 0);
    for (int64_t n = 0; n < nNodes; n++) held[size_t(n)] = (bc[3 * n] | bc[3 * n + 1] | bc[3 * n + 2]) ? 1 : 0;
    std::vector<float> density(density0, density0 + nVox);
    Dev<uint8_t> dHeld(static_cast<size_t>(nNodes));
    dHeld.upload(held.data(), size_t(nNodes));
    Dev<float> dIn(static_cast<size_t>(nVox)), dOut(static_cast<size_t>(nVox));
    auto prune = [&](std::vector<float>& d) {
        dIn.upload(d.data(), size_t(nVox));
        pruneFloatingDevice(dims, dIn.p, dHeld.p, dOut.p, nullptr);
        dOut.download(d.data(), size_t(nVox));
    };
    prune(density);
    // the load on each node, for the lost-load fraction (static_study.cpp:23-32)
    std::vector<double> fmag(static_cast<size_t>(nNodes));
    double ftotal = 0;
    for (int64_t n = 0; n < nNodes; n++) {
        fmag[size_t(n)] = std::sqrt(f[3 * n] * f[3 * n] + f[3 * n + 1] * f[3 * n + 1] + f[3 * n + 2] * f[3 * n + 2]);
        ftotal += fmag[size_t(n)];
    }
    Dev<double> dF(static_cast<size_t>(nDof)), dU(static_cast<size_t>(nDof));
    dF.upload(f, size_t(nDof));
    Dev<float> dDens(static_cast<size_t>(nVox)), dMeasure(static_cast<size_t>(nVox));
    std::vector<float> measure(static_cast<size_t>(nVox)), vm(static_cast<size_t>(nNodes)), p1, p3, nodalHost;
    std::vector<double> u(static_cast<size_t>(nDof));
    BreakReason reason = BREAK_STEP_LIMIT;
    peak = 0;
    bool haveU = false;
    for (int step = 0; step < maxSteps; step++) {
        if (std::none_of(density.begin(), density.end(), [](float d) { return d > 0; })) {
            reason = step > 0 ? BREAK_SEPARATED : BREAK_UNSUPPORTED;
            break;
        }
        const auto t0 = std::chrono::steady_clock::now();
        Solver S(dims, density.data(), nu, bc, 1100, nullptr);
        const HostLevel& L0 = S.hierarchy().levels[0];
        // the lost-load fraction: load on nodes that are no element's corner
        double lost = 0;
        for (int64_t n = 0; n < nNodes; n++)
            if (!(L0.nmask[size_t(n)] & NM_ACTIVE)) lost += fmag[size_t(n)];
        if (L0.nElems == 0 || (ftotal > 0 && lost / ftotal > 0.5)) {
            reason = step > 0 ? BREAK_SEPARATED : BREAK_UNSUPPORTED;
            break;
        }
        ps_solve_opts so;
        ps_solve_opts_default(&so);
        so.tol = 1e-6;  // buildAndSolve (static_study.cpp:79)
        so.max_iter = 3000;
        so.x0 = haveU ? dU.p : nullptr;
        ps_solve_result sr{};
        S.solveDevice(dF.p, so, dU.p, sr);
        ck(cudaDeviceSynchronize(), "break solve");
        if (!sr.converged) {
            reason = BREAK_NOT_CONVERGED;
            break;
        }
        haveU = true;
        dU.download(u.data(), size_t(nDof));
        std::vector<double> uPhys(static_cast<size_t>(nDof));
        const double scale = 1 / (E * h);
        for (int64_t i = 0; i < nDof; i++) uPhys[size_t(i)] = u[size_t(i)] * scale;
        p1.resize(static_cast<size_t>(nNodes));
        p3.resize(static_cast<size_t>(nNodes));
        S.stresses(uPhys.data(), E, h, principal, vm.data(), principal ? p1.data() : nullptr, principal ? p3.data() : nullptr);
        const std::vector<float>& nodal = principal ? p1 : vm;
        // the failure measure of every solved voxel on the device
        {
            Dev<float> dNodal(static_cast<size_t>(nNodes));
            dNodal.upload(nodal.data(), size_t(nNodes));
            dDens.upload(density.data(), size_t(nVox));
            k_break_measure<<<gridOf(nVox, sm), 256>>>(nVox, nx, ny, dDens.p, dNodal.p, dMeasure.p);
            ck(cudaGetLastError(), "measure");
            dMeasure.download(measure.data(), size_t(nVox));
        }
        std::vector<int> solved;
        double smax = 0;
        for (int64_t e = 0; e < nVox; e++)
            if (measure[size_t(e)] >= 0.f) {
                solved.push_back(int(e));
                smax = std::max(smax, double(measure[size_t(e)]));
            }
        if (!(smax > 0)) {
            reason = BREAK_NO_STRESS;
            break;
        }
        BreakStep bs;
        bs.step = step;
        bs.lambda = strength / smax;
        peak = std::max(peak, bs.lambda);
        double dmax = 0;
        for (int64_t n = 0; n < nNodes; n++)
            dmax = std::max(dmax, uPhys[3 * n] * uPhys[3 * n] + uPhys[3 * n + 1] * uPhys[3 * n + 1] + uPhys[3 * n + 2] * uPhys[3 * n + 2]);
        bs.maxDisp = std::sqrt(dmax) * bs.lambda;
        bs.voxels = int(solved.size());
        bs.solveIterations = sr.iterations;
        // the most stressed voxels crack: at most 2 % of n^(2/3), those within 5 % of the peak
        // (static_study.cpp:248-258); stable order by measure, then voxel index
        const size_t cap = std::max<size_t>(1, size_t(std::lround(0.02 * std::pow(double(solved.size()), 2.0 / 3))));
        std::vector<int> cand;
        for (int e : solved)
            if (measure[size_t(e)] >= 0.95 * smax) cand.push_back(e);
        std::stable_sort(cand.begin(), cand.end(), [&](int a, int b) { return measure[size_t(a)] > measure[size_t(b)]; });
        for (int e : cand) {
            if (bs.cracked.size() >= cap) break;
            bs.cracked.push_back(e);
        }
        std::vector<float> next = density;
        for (int e : bs.cracked) next[size_t(e)] = 0;
        std::vector<float> pruned = next;
        prune(pruned);
        for (int64_t e = 0; e < nVox; e++)
            if (next[size_t(e)] > 0 && !(pruned[size_t(e)] > 0)) bs.detached.push_back(int(e));
        density = std::move(pruned);
        bs.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        steps.push_back(std::move(bs));
    }
    std::copy(density.begin(), density.end(), densityOut);
    return reason;
}

}  // namespace psfea
