// Study loops on the device (SIMP topology optimisation, break test): plain C++ interface, CUDA
// inside study.cu.
#pragma once

#include <cstdint>
#include <vector>

#include "ps_fea.h"

namespace psfea {

// a usable CUDA device is present
bool deviceAvailable();

// pruneFloating (voxel_fea.cpp:1086-1119) on device arrays: outDev = densityDev where the voxel's
// 6-connected solid component has a voxel with a held corner node (heldDev: per node), else 0;
// returns the number of solid voxels removed. Stream-ordered; waits for its result.
int pruneFloatingDevice(const int32_t dims[3], const float* densityDev, const uint8_t* heldDev, float* outDev, void* stream);

// native/src/fea/topology.hpp:38-48 and the solve of native/src/fea/study_runner.cpp:403-419
struct TopologyOptions {
    double volFrac = 0.4, penal = 3, rmin = 1.5, move = 0.2, tol = 0.01;
    int maxIter = 40;
    double solveTol = 1e-5;
    int precision = PS_PREC_FP64;
};

struct TopologyStep {
    int it = 0;
    double compliance = 0, volume = 0, change = 0;
    int solveIterations = 0;
    int solveStatus = 0;
    double seconds = 0;
};

// Runs the optimisation; densityOut (nx ny nz) receives the final physical densities (0 outside the
// design domain). Returns the number of iterations recorded in history.
int topologyRun(const int32_t dims[3], const float* fill, const uint8_t* keep, double nu, const uint8_t* bc, const double* f,
                const TopologyOptions& o, float* densityOut, std::vector<TopologyStep>& history);

// native/src/fea/static_study.hpp BreakResult::reason
enum BreakReason { BREAK_STEP_LIMIT = 0, BREAK_SEPARATED = 1, BREAK_UNSUPPORTED = 2, BREAK_NOT_CONVERGED = 3, BREAK_NO_STRESS = 4 };

struct BreakStep {
    int step = 0;
    double lambda = 0, maxDisp = 0;
    int voxels = 0, solveIterations = 0;
    double seconds = 0;
    std::vector<int> cracked, detached;
};

// Runs the break test (native/src/fea/static_study.cpp:199-279); densityOut receives the density
// left after the last step, peak the largest load factor.
BreakReason breakTest(const int32_t dims[3], const float* density, double nu, const uint8_t* bc, const double* f, double E, double h,
                      double strength, bool principal, int maxSteps, std::vector<BreakStep>& steps, float* densityOut, double& peak);

}  // namespace psfea
