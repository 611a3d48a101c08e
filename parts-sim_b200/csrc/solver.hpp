// Device-resident solver for one voxel model (plain C++ interface; CUDA stays inside solver.cu).
#pragma once

#include <cstdint>
#include <memory>

#include "hierarchy.hpp"
#include "ps_fea.h"

namespace psfea {

struct SolverImpl;
struct SolverHandle;
struct BlockBase;

// the configuration an autotune run chose for a model (and what it measured)
struct TuneResult {
    int degree = 2;           // Chebyshev smoother degree per V-cycle half
    int64_t splitLevels = 0;  // bit l: level l's 32-bit tiles leave boundary nodes to the list kernel
    int inner64 = 0;          // the finest level's 64-bit tiles compute boundary nodes in the tile
    int trials = 0;           // solves timed (0: taken from the cache)
    double bestSeconds = 0;   // the chosen configuration's solve time
    double defaultSeconds = 0;  // the configuration before tuning
    int cached = 0;
};

class Solver {
public:
    // builds the hierarchy on the host and uploads it; throws Error
    Solver(const int32_t dims[3], const float* density, double nu, const uint8_t* bc, int64_t coarsestMaxDof, const double* diagAdd);
    // uploads a hierarchy built beforehand (buildHierarchy may run on any host thread)
    explicit Solver(Hierarchy&& hier);
    ~Solver();

    const Hierarchy& hierarchy() const;
    int64_t nDof() const;
    int64_t deviceBytes() const;
    int64_t contextBytes() const;  // device bytes of one solve context (work vectors and state)
    double levelLmax(int l) const;

    // host vectors in/out; returns the outcome status
    ps_status solve(const double* f, const ps_solve_opts& o, double* u, ps_solve_result& res);
    // device vectors in/out (o.x0 is a device pointer)
    ps_status solveDevice(const double* fDev, const ps_solve_opts& o, double* uDev, ps_solve_result& res);
    // nrhs solves on this hierarchy: in blocks of up to 32 right-hand sides whose kernels take the
    // whole block (FP64-Krylov forms), or up to `concurrency` at once on separate streams, each its
    // own context (the FP32-Krylov form, or PSFEA_BATCH_MODE=contexts)
    ps_status solveBatch(int32_t nrhs, const double* f, const ps_solve_opts& o, double* u, ps_solve_result* results, int concurrency);
    // z_k = one V-cycle applied to r_k for nvec dense device vectors (consecutive), in blocks of up
    // to 32; stream-ordered on s (nullptr = the handle's stream)
    void preconditionBlock(int32_t nvec, const double* rDev, double* zDev, void* s);
    // non-blocking solve for a serving loop: begin() enqueues it (f and u stay valid until poll()
    // returns true), poll() moves it on without waiting for the GPU
    void begin(const double* fHost, const ps_solve_opts& o, double* uHost);
    bool poll(ps_solve_result& res);
    void precondition(const double* r, double* z);
    void apply(int level, const double* x, double* y, bool raw);
    void stresses(const double* u, double E, double h, bool principals, float* vm, float* p1, float* p3);
    void reactions(const double* u, const double* f, double R[3]);
    // route all work to the caller's CUDA stream (nullptr = the handle's own)
    void setStream(void* stream);
    // mean device time (ms, CUDA events) of the finest level's operator kernel: 0 = the FP32
    // Chebyshev step of the V-cycle, 1 = the FP64 product of the CG
    double timeKernel(int which, int reps);
    int64_t launches() const;
    // times solves of f (host) to o.tol over smoother degrees 1-4 and the tile-path choices of the
    // tiled levels (coordinate descent: degree first, then each tile flag), keeps the fastest
    // configuration on this handle (solves that leave the degree open use it) and caches it by the
    // model's signature; force: ignore the cache
    TuneResult autotune(const double* f, const ps_solve_opts& o, bool force);
    // y = K x and x.y on the finest level, device pointers, with no allocation (scratch in a
    // static device array); stream-ordered on s (nullptr = the handle's stream), no host sync
    void applyDotStatic(const double* xDev, double* yDev, double* dotDev, void* s);

private:
    BlockBase* blockFor(int nrhs);  // the block context for nrhs right-hand sides (null: none fits)
    std::unique_ptr<SolverImpl> impl_;
    std::unique_ptr<SolverHandle> handle_;
};

// device bytes a Solver over this hierarchy takes (its data and one solve context), for admission
int64_t estimateDeviceBytes(const Hierarchy& H);

}  // namespace psfea
