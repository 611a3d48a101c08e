// Host-side build of the geometric multigrid hierarchy: the level data every device kernel
// reads. The rules follow native/src/fea/voxel_fea.cpp:113-386 and :612-661.
#pragma once

#include <cstdint>
#include <memory>
#include <utility>
#include <vector>

#include "element.hpp"

namespace psfea {

// Voxel word: 0 = empty; bit 31 clear = the float bits of s for an element s * Kb (s > 0);
// bit 31 set = the index of the element's own 24x24 matrix in the low 31 bits.
constexpr uint32_t OWN_BIT = 0x80000000u;

// node mask bits
constexpr uint8_t NM_FIXED0 = 1, NM_FIXED1 = 2, NM_FIXED2 = 4;  // DOF d held, inactive or zero diagonal
constexpr uint8_t NM_ACTIVE = 8;    // the node is a corner of some element
constexpr uint8_t NM_UNIFORM = 16;  // its 8 voxels are the same s * Kb: the 27-point stencil applies

// An allocator whose new elements are left uninitialised: for large host arrays that parallel
// loops fill completely right after allocation (no serial zero fill first)
template <class T>
struct UninitAlloc : std::allocator<T> {
    template <class U>
    struct rebind {
        using other = UninitAlloc<U>;
    };
    UninitAlloc() = default;
    template <class U>
    UninitAlloc(const UninitAlloc<U>&) noexcept {}
    template <class U>
    void construct(U* p) noexcept {
        ::new (static_cast<void*>(p)) U;
    }
    template <class U, class... A>
    void construct(U* p, A&&... a) {
        ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
    }
};

struct HostLevel {
    int nx = 0, ny = 0, nz = 0, NX = 0, NY = 0, NZ = 0;
    int64_t nVox = 0, nNodes = 0, nDof = 0;
    int64_t nElems = 0, nOwn = 0, freeDof = 0;
    std::vector<uint32_t> word;   // per voxel
    std::vector<float, UninitAlloc<float>> own;  // nOwn * 576, row-major 24x24 each (32-bit, as the reference stores them)
    std::vector<int32_t> ownClass;  // per own matrix: equal classes hold bitwise-equal matrices
    double Kb[576];               // the level's uniform element: K0, then the Galerkin sum of 8 children
    double S[27][9];              // Kb assembled into the 27-point stencil: neighbour m = (ox+1) + 3(oy+1) + 9(oz+1), row d, col c
    std::vector<uint8_t> bc;      // per DOF
    std::vector<double> diagAdd;  // per DOF, or empty
    std::vector<double, UninitAlloc<double>> invDiag;  // per DOF, 0 where fixed
    std::vector<uint8_t, UninitAlloc<uint8_t>> nmask;  // per node
    std::vector<int32_t> boundary;  // active nodes without NM_UNIFORM, increasing
    double lmax = 0;              // largest eigenvalue estimate of D^-1 K (smoother), 0 = not yet

    int64_t node(int i, int j, int k) const { return i + int64_t(NX) * (j + int64_t(NY) * k); }
    int64_t voxel(int i, int j, int k) const { return i + int64_t(nx) * (j + int64_t(ny) * k); }
    bool fixedDof(int64_t i) const { return (nmask[i / 3] >> (i % 3)) & 1; }
};

struct Hierarchy {
    HexElement el;
    double nu = 0.3;
    std::vector<HostLevel> levels;
    // coarsest level: free DOF list (level DOF index of dense row q) and the dense inverse of its
    // matrix in FP64 from the regularised Cholesky factor; empty = 40 damped Jacobi sweeps instead
    std::vector<int32_t> coarseDof;
    std::vector<double> coarseInv;
    std::vector<double> coarseChol;  // lower factor, row-major (kept for the exact one-level case)
    int64_t coarseM = 0;
    bool hasFactor() const { return !coarseInv.empty(); }
};

// Computes the own Galerkin matrices of a coarse level somewhere other than the host loop (the
// device engine of galerkin.cu): every own matrix o of C (coarse voxel ownVox[o]) as the host loop
// computes it, bitwise (the same FP64 products and sums in the same order, rounded once to 32 bits).
// M: the 8 child products P_c^T F.Kb P_c. coarsen() hands a level over when its classes of equal
// child patterns number at least minClasses() (graded grids: every matrix distinct); lattices with
// a few hundred classes stay on the host.
struct GalerkinEngine {
    virtual ~GalerkinEngine() = default;
    virtual int64_t minClasses() const = 0;
    virtual void computeOwn(const HostLevel& F, const HostLevel& C, const std::vector<int64_t>& ownVox, const double (*M)[576],
                            float* out) = 0;
};

// the device engine on the current CUDA device (galerkin.cu), taking levels of at least
// minClasses classes (PSFEA_DEVICE_GALERKIN_MIN overrides); throws Error(PS_ENODEV / PS_ECUDA)
std::unique_ptr<GalerkinEngine> makeDeviceGalerkin(int64_t minClasses = 4096);

// Validates the inputs (Error(PS_EINVAL) with the reference's messages) and builds everything;
// with an engine, the own matrices of graded coarse levels come from it.
Hierarchy buildHierarchy(const int32_t dims[3], const float* density, double nu, const uint8_t* bc, int64_t coarsestMaxDof,
                         const double* diagAdd, GalerkinEngine* engine = nullptr);

// tridiagonal (a, b) largest eigenvalue by Sturm-count bisection (voxel_fea.cpp:506-530)
double tridiagonalMax(const std::vector<double>& a, const std::vector<double>& b);

// degree-2 Chebyshev coefficients on [0.1, 1.15] * lmax (voxel_fea.cpp:692-701)
void chebyshevCoefficients(double lmax, double& first, double& c1, double& c2);

}  // namespace psfea
