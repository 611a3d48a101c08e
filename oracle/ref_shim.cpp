// ORACLE — test infrastructure only. A C ABI over the reference's own solver class
// (native/src/fea/voxel_fea.hpp:130-189), compiled together with the reference's sources by
// oracle/Makefile into oracle/_ref/libpsref.so. It exposes the same entry points as
// oracle/psoracle.cpp (prefix ref_ instead of orc_) so the tests can run either side by side.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <vector>

#include <memory>

#include "fea/hex8.hpp"
#include "fea/topology.hpp"
#include "fea/voxel_fea.hpp"

extern "C" {

static void setErr(char* err, int len, const char* msg) {
    if (err && len > 0) std::snprintf(err, size_t(len), "%s", msg);
}

void* ref_create(const int32_t dims[3], const float* density, double nu, const uint8_t* bc, int64_t coarsest, const double* diag_add, char* err, int errlen) {
    try {
        const int64_t nE = int64_t(dims[0]) * dims[1] * dims[2];
        const int64_t nDof = 3 * int64_t(dims[0] + 1) * (dims[1] + 1) * (dims[2] + 1);
        std::vector<float> d(density, density + (nE > 0 ? nE : 0));
        std::vector<uint8_t> b(bc, bc + (nDof > 0 ? nDof : 0));
        std::vector<double> da;
        if (diag_add) da.assign(diag_add, diag_add + nDof);
        return new ps::VoxelFEA({dims[0], dims[1], dims[2]}, d, nu, b, coarsest, diag_add ? &da : nullptr);
    } catch (const std::exception& e) {
        setErr(err, errlen, e.what());
        return nullptr;
    }
}
void ref_destroy(void* h) { delete static_cast<ps::VoxelFEA*>(h); }
int ref_num_levels(void* h) { return int(static_cast<ps::VoxelFEA*>(h)->levels.size()); }
void ref_level_info(void* h, int l, int64_t* out) {
    auto* F = static_cast<ps::VoxelFEA*>(h);
    const auto& L = F->levels[l];
    out[0] = L.nx; out[1] = L.ny; out[2] = L.nz; out[3] = L.nNodes; out[4] = L.nDof; out[5] = L.freeDof;
    out[6] = int64_t(L.elems.size()); out[7] = int64_t(L.K.size() / 576); out[8] = F->coarse.m;
}
void ref_level_fixed(void* h, int l, uint8_t* out) { auto& L = static_cast<ps::VoxelFEA*>(h)->levels[l]; std::memcpy(out, L.fixed.data(), L.fixed.size()); }
void ref_level_active(void* h, int l, uint8_t* out) { auto& L = static_cast<ps::VoxelFEA*>(h)->levels[l]; std::memcpy(out, L.activeNode.data(), L.activeNode.size()); }
void ref_level_kb(void* h, int l, double* out) { std::memcpy(out, static_cast<ps::VoxelFEA*>(h)->levels[l].Kb.data(), 576 * 8); }
void ref_level_elems(void* h, int l, int32_t* out) { auto& L = static_cast<ps::VoxelFEA*>(h)->levels[l]; for (size_t e = 0; e < L.elems.size(); e++) out[e] = L.elems[e]; }
void ref_level_kidx(void* h, int l, int32_t* out) {
    auto& L = static_cast<ps::VoxelFEA*>(h)->levels[l];
    for (size_t e = 0; e < L.elems.size(); e++) out[e] = L.kIdx.empty() ? -1 : L.kIdx[e];
}
void ref_level_rho(void* h, int l, double* out) { auto& L = static_cast<ps::VoxelFEA*>(h)->levels[l]; std::memcpy(out, L.rho.data(), L.rho.size() * 8); }
void ref_level_own(void* h, int l, float* out) {
    auto& L = static_cast<ps::VoxelFEA*>(h)->levels[l];
    const size_t n = L.K.size() / 576 * 576;
    if (n) std::memcpy(out, L.K.data(), n * 4);
}
void ref_level_invdiag(void* h, int l, double* out) { auto& L = static_cast<ps::VoxelFEA*>(h)->levels[l]; std::memcpy(out, L.invDiag.data(), L.invDiag.size() * 8); }
void ref_prepare(void* h) { static_cast<ps::VoxelFEA*>(h)->prepareSmoothers(); }
double ref_level_lmax(void* h, int l) { return static_cast<ps::VoxelFEA*>(h)->levels[l].lmax; }
void ref_set_lmax(void* h, int l, double v) { auto& L = static_cast<ps::VoxelFEA*>(h)->levels[l]; L.lmax = v; L.omega = 1.2 / (v * 1.05); }
void ref_apply(void* h, int l, const double* x, double* y, int raw) { static_cast<ps::VoxelFEA*>(h)->apply(l, x, y, raw != 0); }
void ref_precondition(void* h, const double* r, double* z) { static_cast<ps::VoxelFEA*>(h)->precondition(r, z); }
void ref_vcycle32(void* h, int l, const float* r, float* z) {
    auto* F = static_cast<ps::VoxelFEA*>(h);
    F->prepareSmoothers();
    auto& L = F->levels[l];
    std::memcpy(L.r.data(), r, L.r.size() * 4);
    F->vcycle(l);
    std::memcpy(z, L.z.data(), L.z.size() * 4);
}
void ref_coarse_factor(void* h, double* out) { auto* F = static_cast<ps::VoxelFEA*>(h); std::memcpy(out, F->coarse.A.data(), F->coarse.A.size() * 8); }
int ref_solve(void* h, const double* f, double tol, int max_iter, const double* x0, double* u, int32_t* iters, double* residual, int32_t* converged,
              char* err, int errlen) {
    try {
        auto* F = static_cast<ps::VoxelFEA*>(h);
        const int64_t n = F->nDof();
        std::vector<double> fv(f, f + n), xv;
        ps::SolveOptions o;
        o.tol = tol;
        o.maxIter = max_iter;
        if (x0) { xv.assign(x0, x0 + n); o.x0 = &xv; }
        const auto r = F->solve(fv, o);
        std::memcpy(u, r.u.data(), size_t(n) * 8);
        *iters = r.iterations;
        *residual = r.residual;
        *converged = r.converged;
        return 0;
    } catch (const std::exception& e) {
        setErr(err, errlen, e.what());
        return 1;
    }
}
void ref_stresses(void* h, const double* u, double E, double hh, int principals, float* vm, float* p1, float* p3) {
    auto* F = static_cast<ps::VoxelFEA*>(h);
    std::vector<double> uv(u, u + F->nDof());
    const auto s = F->stresses(uv, E, hh, principals != 0);
    std::memcpy(vm, s.nodeVM.data(), s.nodeVM.size() * 4);
    if (principals) {
        std::memcpy(p1, s.nodeP1.data(), s.nodeP1.size() * 4);
        std::memcpy(p3, s.nodeP3.data(), s.nodeP3.size() * 4);
    }
}
void ref_reactions(void* h, const double* u, const double* f, double* R) {
    auto* F = static_cast<ps::VoxelFEA*>(h);
    std::vector<double> uv(u, u + F->nDof()), fv;
    if (f) fv.assign(f, f + F->nDof());
    const auto r = F->reactions(uv, f ? &fv : nullptr);
    R[0] = r[0]; R[1] = r[1]; R[2] = r[2];
}
int ref_element(double nu, int modes, double* K, double* cornerStress, double* gaussB, char* err, int errlen) {
    try {
        const auto el = ps::hexElement(nu, modes != 0);
        std::memcpy(K, el.K.data(), 576 * 8);
        if (cornerStress)
            for (int a = 0; a < 8; a++) std::memcpy(cornerStress + 144 * a, el.cornerStress[a].data(), 144 * 8);
        if (gaussB)
            for (int a = 0; a < 8; a++) std::memcpy(gaussB + 144 * a, el.gaussB[a].data(), 144 * 8);
        return 0;
    } catch (const std::exception& e) {
        setErr(err, errlen, e.what());
        return 1;
    }
}
int ref_prune(const int32_t dims[3], const float* density, const uint8_t* heldNode, float* out) {
    const int64_t nE = int64_t(dims[0]) * dims[1] * dims[2], nN = int64_t(dims[0] + 1) * (dims[1] + 1) * (dims[2] + 1);
    std::vector<float> d(density, density + nE);
    std::vector<uint8_t> held(heldNode, heldNode + nN);
    const auto r = ps::pruneFloating({dims[0], dims[1], dims[2]}, d, held);
    std::memcpy(out, r.density.data(), size_t(nE) * 4);
    return r.removed;
}

// optimizeTopology (native/src/fea/topology.cpp:103-183) with the solve of runTopology
// (native/src/fea/study_runner.cpp:403-419: a fresh VoxelFEA per iteration, coarsest 1100 DOFs,
// tol solveTol, 3000 iterations, warm start). hist: maxIter rows of (it, compliance, volume, change).
int ref_topology(const int32_t dims[3], const float* fill, const uint8_t* keep, double nu, const uint8_t* bc, const double* f, double volFrac,
                 double penal, double rmin, double move, double tol, int maxIter, double solveTol, float* densityOut, double* hist, int* nHist,
                 char* err, int errlen) {
    try {
        const int64_t nE = int64_t(dims[0]) * dims[1] * dims[2];
        const int64_t nDof = 3 * int64_t(dims[0] + 1) * (dims[1] + 1) * (dims[2] + 1);
        ps::TopologyOptions o;
        o.dims = {dims[0], dims[1], dims[2]};
        o.fill.assign(fill, fill + nE);
        o.keep.assign(size_t(nE), 0);
        if (keep) o.keep.assign(keep, keep + nE);
        o.volFrac = volFrac;
        o.penal = penal;
        o.rmin = rmin;
        o.move = move;
        o.tol = tol;
        o.maxIter = maxIter;
        const std::vector<uint8_t> bcv(bc, bc + nDof);
        const std::vector<double> fv(f, f + nDof);
        std::unique_ptr<ps::VoxelFEA> fea;
        o.solve = [&](const std::vector<float>& density, const std::vector<double>* x0) {
            fea = std::make_unique<ps::VoxelFEA>(o.dims, density, nu, bcv, 1100);
            ps::SolveOptions so;
            so.tol = solveTol;
            so.maxIter = 3000;
            so.x0 = x0;
            auto sol = fea->solve(fv, so);
            return ps::TopologySolve{std::move(sol.u), fv, fea.get()};
        };
        const auto res = ps::optimizeTopology(o);
        std::memcpy(densityOut, res.density.data(), size_t(nE) * 4);
        *nHist = int(res.history.size());
        for (size_t k = 0; k < res.history.size(); k++) {
            hist[4 * k] = res.history[k].it;
            hist[4 * k + 1] = res.history[k].compliance;
            hist[4 * k + 2] = res.history[k].volume;
            hist[4 * k + 3] = res.history[k].change;
        }
        return 0;
    } catch (const std::exception& e) {
        setErr(err, errlen, e.what());
        return 1;
    }
}

}  // extern "C"
