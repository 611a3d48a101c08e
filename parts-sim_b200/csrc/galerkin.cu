// Galerkin coarsening on the device: the own matrices of a coarse level, P_c^T K_c P_c summed over
// the 8 children of each coarse voxel (the rule of native/src/fea/voxel_fea.cpp:309-354, whose
// galerkinAdd at :86-111 forms the same two-stage product T = K P_c, then P_c^T T).
//
// Graded grids (SIMP densities) share no class of equal child patterns, so the host computes every
// coarse matrix of every level on every rebuild, and a topology loop rebuilds its model once per
// iteration (native/src/fea/study_runner.cpp:403-419). Here one CTA takes one coarse voxel at a
// time: 192 threads own 3 of its 576 entries each and accumulate them in FP64 registers over the
// children; an own child's matrix is staged in shared memory and its T = K P_c formed there. The
// products and sums are the host's, in the host's order, with no fused multiply-adds (__dmul_rn /
// __dadd_rn), rounded once to 32 bits: the matrices come out bitwise equal to the host loop's.
// The level just computed stays on the device as the fine level of the next coarsening.
#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "element.hpp"
#include "hierarchy.hpp"
#include "host_util.hpp"

namespace psfea {

namespace dev {

constexpr int GT = 192;  // threads per coarse voxel: 3 of the 576 entries each

// cw: the 8 child words of each own coarse voxel (0 empty, float bits of s, OWN_BIT | fine own
// index); fineOwn: the fine level's own matrices (32-bit); M: the 8 child products of the fine
// uniform element (FP64); W: child weights [c][a][b]; out: nOwn x 576 floats
__global__ void __launch_bounds__(GT) k_galerkin(long long nOwn, const uint32_t* __restrict__ cw, const float* __restrict__ fineOwn,
                                                 const double* __restrict__ M, const double* __restrict__ W, float* __restrict__ out) {
    __shared__ double sW[512];
    __shared__ double sK[576];
    __shared__ double sT[576];
    __shared__ uint32_t sw[8];
    for (int i = threadIdx.x; i < 512; i += GT) sW[i] = W[i];
    for (long long o = blockIdx.x; o < nOwn; o += gridDim.x) {
        __syncthreads();  // the previous voxel's reads of sw, sK and sT are done (and sW is written)
        if (threadIdx.x < 8) sw[threadIdx.x] = cw[o * 8 + threadIdx.x];
        __syncthreads();
        double acc[3] = {0.0, 0.0, 0.0};
        for (int c = 0; c < 8; c++) {
            const uint32_t w = sw[c];  // the same in every thread: the branches below are uniform
            if (!w) continue;
            if (w & 0x80000000u) {
                const float* src = fineOwn + (long long)(w & 0x7fffffffu) * 576;
                for (int u = threadIdx.x; u < 576; u += GT) sK[u] = double(__ldg(src + u));
                __syncthreads();
                // T = K P_c: entry (r, 3 b + e) sums K[r][3 a + e] W[c][a][b] over a in increasing
                // order, zero weights skipped
                for (int u = threadIdx.x; u < 576; u += GT) {
                    const int r = u / 24, col = u - 24 * r, b = col / 3, e = col - 3 * b;
                    double t = 0.0;
#pragma unroll
                    for (int a = 0; a < 8; a++) {
                        const double wt = sW[(c * 8 + a) * 8 + b];
                        if (wt != 0.0) t = __dadd_rn(t, __dmul_rn(sK[r * 24 + 3 * a + e], wt));
                    }
                    sT[u] = t;
                }
                __syncthreads();
                // out += P_c^T T: entry (3 b + d, q) adds W[c][a][b] T[3 a + d][q] over a in order
#pragma unroll
                for (int e = 0; e < 3; e++) {
                    const int u = threadIdx.x + GT * e, R = u / 24, q = u - 24 * R, b = R / 3, d = R - 3 * b;
#pragma unroll
                    for (int a = 0; a < 8; a++) {
                        const double wt = sW[(c * 8 + a) * 8 + b];
                        if (wt != 0.0) acc[e] = __dadd_rn(acc[e], __dmul_rn(wt, sT[(3 * a + d) * 24 + q]));
                    }
                }
                __syncthreads();  // sK and sT are rewritten by the next own child
            } else {
                const double s = double(__uint_as_float(w));
#pragma unroll
                for (int e = 0; e < 3; e++) acc[e] = __dadd_rn(acc[e], __dmul_rn(s, __ldg(M + c * 576 + threadIdx.x + GT * e)));
            }
        }
#pragma unroll
        for (int e = 0; e < 3; e++) out[o * 576 + threadIdx.x + GT * e] = __double2float_rn(acc[e]);
    }
}

}  // namespace dev

namespace {

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) throw Error(PS_ENODEV, std::string(what) + ": " + cudaGetErrorString(e));
        throw Error(PS_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

// interpolation weight of coarse corner b at corner a of the fine child in position c (the rule of
// the host build: 1 or 1/2 per axis, exact in FP64)
double childWeight(int c, int a, int b) {
    double w = 1;
    for (int d = 0; d < 3; d++) {
        const double s = (((c >> d) & 1) + CORNER_XYZ[a][d]) * 0.5;
        w *= CORNER_XYZ[b][d] ? s : 1 - s;
    }
    return w;
}

class DeviceGalerkin final : public GalerkinEngine {
public:
    explicit DeviceGalerkin(int64_t minClasses) : min_(minClasses) {
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
            cudaGetLastError();
            throw Error(PS_ENODEV, "no CUDA device is available");
        }
        ck(cudaGetDevice(&dev_), "cudaGetDevice");
        ck(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, dev_), "attribute");
        ck(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking), "stream");
        if (const char* e = std::getenv("PSFEA_DEVICE_GALERKIN_MIN")) min_ = std::atoll(e);
        std::vector<double> W(512);
        for (int c = 0; c < 8; c++)
            for (int a = 0; a < 8; a++)
                for (int b = 0; b < 8; b++) W[size_t((c * 8 + a) * 8 + b)] = childWeight(c, a, b);
        dW_ = alloc<double>(512);
        dM_ = alloc<double>(8 * 576);
        ck(cudaMemcpyAsync(dW_, W.data(), 512 * sizeof(double), cudaMemcpyHostToDevice, st_), "upload");
        ck(cudaStreamSynchronize(st_), "galerkin setup");
    }
    ~DeviceGalerkin() override {
        if (!st_) return;
        for (void* p : {static_cast<void*>(dW_), static_cast<void*>(dM_), static_cast<void*>(last_)})
            if (p) cudaFreeAsync(p, st_);
        cudaStreamSynchronize(st_);
        cudaStreamDestroy(st_);
    }
    int64_t minClasses() const override { return min_; }

    void computeOwn(const HostLevel& F, const HostLevel& C, const std::vector<int64_t>& ownVox, const double (*M)[576], float* out) override {
        int cur = -1;
        ck(cudaGetDevice(&cur), "cudaGetDevice");
        if (cur != dev_) throw Error(PS_EINVAL, "the Galerkin engine was created on another device");
        const int64_t nOwn = int64_t(ownVox.size());
        // the 8 child words of every own coarse voxel
        std::vector<uint32_t> cw(size_t(nOwn) * 8);
        parallelFor(nOwn, [&](int64_t o0, int64_t o1) {
            for (int64_t o = o0; o < o1; o++) {
                const int64_t v = ownVox[size_t(o)];
                const int I = int(v % C.nx), J = int((v / C.nx) % C.ny), K = int(v / (int64_t(C.nx) * C.ny));
                for (int c = 0; c < 8; c++) {
                    const int i = 2 * I + (c & 1), j = 2 * J + ((c >> 1) & 1), k = 2 * K + (c >> 2);
                    cw[size_t(o * 8 + c)] = (i >= F.nx || j >= F.ny || k >= F.nz) ? 0u : F.word[size_t(F.voxel(i, j, k))];
                }
            }
        }, 4096);
        // the fine own matrices: still on the device when this engine computed them (the previous
        // level), uploaded otherwise
        float* fine = nullptr;
        bool fineIsLast = false;
        if (F.nOwn > 0) {
            if (last_ && lastN_ == F.nOwn && lastDims_[0] == F.nx && lastDims_[1] == F.ny && lastDims_[2] == F.nz) {
                fine = last_;
                fineIsLast = true;
            } else {
                fine = alloc<float>(size_t(F.nOwn) * 576);
                ck(cudaMemcpyAsync(fine, F.own.data(), size_t(F.nOwn) * 576 * sizeof(float), cudaMemcpyHostToDevice, st_), "upload");
            }
        }
        uint32_t* dcw = alloc<uint32_t>(cw.size());
        float* dOut = alloc<float>(size_t(nOwn) * 576);
        ck(cudaMemcpyAsync(dcw, cw.data(), cw.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st_), "upload");
        ck(cudaMemcpyAsync(dM_, M, 8 * 576 * sizeof(double), cudaMemcpyHostToDevice, st_), "upload");
        const int grid = int(std::max<int64_t>(1, std::min<int64_t>(nOwn, int64_t(sms_) * 10)));
        dev::k_galerkin<<<grid, dev::GT, 0, st_>>>(nOwn, dcw, fine, dM_, dW_, dOut);
        ck(cudaGetLastError(), "k_galerkin");
        ck(cudaMemcpyAsync(out, dOut, size_t(nOwn) * 576 * sizeof(float), cudaMemcpyDeviceToHost, st_), "download");
        ck(cudaFreeAsync(dcw, st_), "free");
        if (fine && !fineIsLast) ck(cudaFreeAsync(fine, st_), "free");
        if (last_) ck(cudaFreeAsync(last_, st_), "free");
        ck(cudaStreamSynchronize(st_), "k_galerkin");
        last_ = dOut;  // the next coarsening's fine level
        lastN_ = nOwn;
        lastDims_[0] = C.nx;
        lastDims_[1] = C.ny;
        lastDims_[2] = C.nz;
        launches_++;
    }

private:
    template <class T>
    T* alloc(size_t n) {
        void* p = nullptr;
        ck(cudaMallocAsync(&p, std::max<size_t>(n, 1) * sizeof(T), st_), "cudaMallocAsync");
        return static_cast<T*>(p);
    }
    int dev_ = 0, sms_ = 148;
    cudaStream_t st_ = nullptr;
    int64_t min_;
    double* dW_ = nullptr;
    double* dM_ = nullptr;
    float* last_ = nullptr;  // own matrices of the level computed last
    int64_t lastN_ = 0;
    int lastDims_[3] = {0, 0, 0};
    int64_t launches_ = 0;
};

}  // namespace

std::unique_ptr<GalerkinEngine> makeDeviceGalerkin(int64_t minClasses) {
    return std::unique_ptr<GalerkinEngine>(new DeviceGalerkin(minClasses));
}

}  // namespace psfea
