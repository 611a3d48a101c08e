// The C ABI of include/ps_fea.h: validation with the reference's messages, exceptions mapped to
// status codes, and the per-thread last-error string.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "element.hpp"
#include "host_util.hpp"
#include "ps_fea.h"
#include "solver.hpp"
#include "study.hpp"

struct ps_fea {
    psfea::Solver solver;
    ps_fea(const int32_t dims[3], const float* density, double nu, const uint8_t* bc, int64_t coarsest, const double* diagAdd)
        : solver(dims, density, nu, bc, coarsest, diagAdd) {}
};

namespace {

thread_local std::string lastError;

ps_status fail(ps_status s, const std::string& msg) {
    lastError = msg;
    return s;
}

template <class F>
ps_status guarded(F&& fn) {
    try {
        lastError.clear();
        return fn();
    } catch (const psfea::Error& e) {
        return fail(e.status, e.what());
    } catch (const std::bad_alloc&) {
        return fail(PS_EOOM, "host memory exhausted");
    } catch (const std::exception& e) {
        return fail(PS_ECUDA, e.what());
    }
}

ps_solve_opts resolve(const ps_solve_opts* o) {
    ps_solve_opts r;
    ps_solve_opts_default(&r);
    if (o) r = *o;
    return r;
}

}  // namespace

extern "C" {

void ps_solve_opts_default(ps_solve_opts* o) {
    if (!o) return;
    o->tol = 1e-6;
    o->max_iter = 500;
    o->precision = PS_PREC_FP64;
    o->x0 = nullptr;
    o->cancel = nullptr;
    o->time_limit_s = 0;
    o->smoother_degree = 0;
}

const char* ps_last_error(void) { return lastError.c_str(); }

ps_status ps_fea_create(const int32_t dims[3], const float* density, double nu, const uint8_t* bc, int64_t coarsest_max_dof,
                        const double* diag_add, ps_fea_t** out) {
    return guarded([&] {
        if (!out) return fail(PS_EINVAL, "out is NULL");
        *out = nullptr;
        if (!dims) return fail(PS_EINVAL, "The structural grid must have three positive dimensions.");
        *out = new ps_fea(dims, density, nu, bc, coarsest_max_dof, diag_add);
        return PS_OK;
    });
}

void ps_fea_destroy(ps_fea_t* h) { delete h; }

ps_status ps_fea_solve(ps_fea_t* h, const double* f, const ps_solve_opts* opts, double* u_out, ps_solve_result* result) {
    return guarded([&] {
        if (!h || !f || !u_out) return fail(PS_EINVAL, "Force or displacement vector has the wrong size.");
        const ps_solve_opts o = resolve(opts);
        if (!(o.tol >= 0) || o.max_iter < 0 || (o.precision < PS_PREC_FP64 || o.precision > PS_PREC_HALF) || o.smoother_degree < 0 ||
            o.smoother_degree > 8)
            return fail(PS_EINVAL, "invalid solve options");
        ps_solve_result r{};
        const ps_status s = h->solver.solve(f, o, u_out, r);
        if (result) *result = r;
        return s;
    });
}

ps_status ps_fea_solve_dev(ps_fea_t* h, const double* f_dev, const ps_solve_opts* opts, double* u_dev, ps_solve_result* result) {
    return guarded([&] {
        if (!h || !f_dev || !u_dev) return fail(PS_EINVAL, "Force or displacement vector has the wrong size.");
        const ps_solve_opts o = resolve(opts);
        if (!(o.tol >= 0) || o.max_iter < 0 || (o.precision < PS_PREC_FP64 || o.precision > PS_PREC_HALF) || o.smoother_degree < 0 ||
            o.smoother_degree > 8)
            return fail(PS_EINVAL, "invalid solve options");
        ps_solve_result r{};
        const ps_status s = h->solver.solveDevice(f_dev, o, u_dev, r);
        if (result) *result = r;
        return s;
    });
}

ps_status ps_fea_solve_batch(ps_fea_t* h, int32_t nrhs, const double* f, const ps_solve_opts* opts, double* u_out, ps_solve_result* results) {
    return guarded([&] {
        if (!h || !f || !u_out || nrhs < 0) return fail(PS_EINVAL, "Force or displacement vector has the wrong size.");
        const ps_solve_opts base = resolve(opts);
        if (!(base.tol >= 0) || base.max_iter < 0 || (base.precision < PS_PREC_FP64 || base.precision > PS_PREC_HALF) ||
            base.smoother_degree < 0 || base.smoother_degree > 8)
            return fail(PS_EINVAL, "invalid solve options");
        if (nrhs == 0) return PS_OK;
        int concurrency = 2;  // concurrent solve contexts; two measured best on a B200 (each solve already fills the GPU)
        if (const char* e = std::getenv("PSFEA_BATCH_CONCURRENCY")) concurrency = std::max(1, std::atoi(e));
        return h->solver.solveBatch(nrhs, f, base, u_out, results, concurrency);
    });
}

ps_status ps_fea_precondition(ps_fea_t* h, const double* r, double* z) {
    return guarded([&] {
        if (!h || !r || !z) return fail(PS_EINVAL, "NULL vector");
        h->solver.precondition(r, z);
        return PS_OK;
    });
}

void ps_topology_opts_default(ps_topology_opts* o) {
    if (!o) return;
    const psfea::TopologyOptions d;
    o->vol_frac = d.volFrac;
    o->penal = d.penal;
    o->rmin = d.rmin;
    o->move = d.move;
    o->tol = d.tol;
    o->max_iter = d.maxIter;
    o->solve_tol = d.solveTol;
    o->precision = d.precision;
}

ps_status ps_topology_run(const int32_t dims[3], const float* fill, const uint8_t* keep, double nu, const uint8_t* bc, const double* f,
                          const ps_topology_opts* opts, float* density_out, ps_topology_step* history, int32_t* n_steps) {
    return guarded([&] {
        if (!dims || !fill || !bc || !f || !density_out) return fail(PS_EINVAL, "NULL argument");
        ps_topology_opts o;
        ps_topology_opts_default(&o);
        if (opts) o = *opts;
        if (!(o.vol_frac > 0 && o.vol_frac <= 1) || !(o.penal >= 1) || !(o.rmin > 0) || !(o.move > 0) || o.max_iter < 0 || !(o.solve_tol > 0) ||
            o.precision < PS_PREC_FP64 || o.precision > PS_PREC_HALF)
            return fail(PS_EINVAL, "invalid topology options");
        if (!psfea::deviceAvailable()) return fail(PS_ENODEV, "no CUDA device is available");
        psfea::TopologyOptions to;
        to.volFrac = o.vol_frac;
        to.penal = o.penal;
        to.rmin = o.rmin;
        to.move = o.move;
        to.tol = o.tol;
        to.maxIter = o.max_iter;
        to.solveTol = o.solve_tol;
        to.precision = o.precision;
        std::vector<psfea::TopologyStep> hist;
        psfea::topologyRun(dims, fill, keep, nu, bc, f, to, density_out, hist);
        for (size_t k = 0; k < hist.size(); k++)
            if (history)
                history[k] = ps_topology_step{hist[k].it, hist[k].solveIterations, hist[k].solveStatus, hist[k].compliance, hist[k].volume,
                                              hist[k].change, hist[k].seconds};
        if (n_steps) *n_steps = int32_t(hist.size());
        return PS_OK;
    });
}

ps_status ps_prune_floating_dev(const int32_t dims[3], const float* density_dev, const uint8_t* held_dev, float* out_dev, int32_t* removed,
                                void* cuda_stream) {
    return guarded([&] {
        if (!dims || !density_dev || !held_dev || !out_dev) return fail(PS_EINVAL, "NULL argument");
        if (!psfea::deviceAvailable()) return fail(PS_ENODEV, "no CUDA device is available");
        const int r = psfea::pruneFloatingDevice(dims, density_dev, held_dev, out_dev, cuda_stream);
        if (removed) *removed = r;
        return PS_OK;
    });
}

ps_status ps_break_test(const int32_t dims[3], const float* density, double nu, const uint8_t* bc, const double* f, double E, double h,
                        double strength, int32_t principal, int32_t max_steps, ps_break_step* steps, int32_t* n_steps, int32_t* cracked,
                        int64_t cracked_cap, float* density_out, double* peak, int32_t* reason) {
    return guarded([&] {
        if (!dims || !density || !bc || !f || !density_out || max_steps < 0) return fail(PS_EINVAL, "NULL argument");
        if (!(E > 0) || !(h > 0)) return fail(PS_EINVAL, "E and h must be positive");
        if (!(strength > 0)) return fail(PS_EINVAL, "Failure strength must be positive.");
        if (!psfea::deviceAvailable()) return fail(PS_ENODEV, "no CUDA device is available");
        std::vector<psfea::BreakStep> st;
        double pk = 0;
        const psfea::BreakReason why =
            psfea::breakTest(dims, density, nu, bc, f, E, h, strength, principal != 0, max_steps, st, density_out, pk);
        int64_t at = 0;
        for (size_t k = 0; k < st.size(); k++) {
            if (steps)
                steps[k] = ps_break_step{st[k].step, st[k].voxels, st[k].solveIterations, int32_t(st[k].cracked.size()),
                                         int32_t(st[k].detached.size()), st[k].lambda, st[k].maxDisp, st[k].seconds};
            for (int e : st[k].cracked)
                if (cracked && at < cracked_cap) cracked[at++] = e;
        }
        if (n_steps) *n_steps = int32_t(st.size());
        if (peak) *peak = pk;
        if (reason) *reason = int32_t(why);
        return PS_OK;
    });
}

namespace {
void toC(const psfea::TuneResult& t, int64_t coarsest, ps_tune_result* out) {
    if (!out) return;
    out->smoother_degree = t.degree;
    out->inner64 = t.inner64;
    out->split_levels = t.splitLevels;
    out->coarsest_max_dof = coarsest;
    out->trials = t.trials;
    out->cached = t.cached;
    out->best_seconds = t.bestSeconds;
    out->default_seconds = t.defaultSeconds;
}
bool validOpts(const ps_solve_opts& o) {
    return o.tol >= 0 && o.max_iter >= 0 && o.precision >= PS_PREC_FP64 && o.precision <= PS_PREC_HALF && o.smoother_degree >= 0 &&
           o.smoother_degree <= 8;
}
}  // namespace

ps_status ps_fea_autotune(ps_fea_t* h, const double* f, const ps_solve_opts* opts, int32_t flags, ps_tune_result* out) {
    return guarded([&] {
        if (!h || !f) return fail(PS_EINVAL, "NULL argument");
        const ps_solve_opts o = resolve(opts);
        if (!validOpts(o)) return fail(PS_EINVAL, "invalid solve options");
        toC(h->solver.autotune(f, o, (flags & PS_TUNE_FORCE) != 0), 0, out);
        return PS_OK;
    });
}

ps_status ps_fea_create_tuned(const int32_t dims[3], const float* density, double nu, const uint8_t* bc, const double* diag_add,
                              const double* f, const ps_solve_opts* opts, int32_t flags, ps_tune_result* out, ps_fea_t** handle) {
    return guarded([&] {
        if (!handle || !f) return fail(PS_EINVAL, "NULL argument");
        *handle = nullptr;
        if (!dims) return fail(PS_EINVAL, "The structural grid must have three positive dimensions.");
        const ps_solve_opts o = resolve(opts);
        if (!validOpts(o)) return fail(PS_EINVAL, "invalid solve options");
        ps_fea_t* best = nullptr;
        psfea::TuneResult bestT;
        int64_t bestC = 0;
        int32_t levelsSeen[3] = {-1, -1, -1};
        const int64_t depths[3] = {300, 1100, 3000};
        for (int c = 0; c < 3; c++) {
            auto* cand = new ps_fea(dims, density, nu, bc, depths[c], diag_add);
            const int32_t nl = int32_t(cand->solver.hierarchy().levels.size());
            bool same = false;
            for (int k = 0; k < c; k++) same = same || levelsSeen[k] == nl;  // the same hierarchy as a depth already timed
            levelsSeen[c] = nl;
            if (same) {
                delete cand;
                continue;
            }
            const psfea::TuneResult t = cand->solver.autotune(f, o, (flags & PS_TUNE_FORCE) != 0);
            if (!best || t.bestSeconds < bestT.bestSeconds) {
                delete best;
                best = cand;
                bestT = t;
                bestC = depths[c];
            } else {
                delete cand;
            }
        }
        toC(bestT, bestC, out);
        *handle = best;
        return PS_OK;
    });
}

ps_status ps_fea_precondition_block(ps_fea_t* h, int32_t nvec, const double* r_dev, double* z_dev, void* cuda_stream) {
    return guarded([&] {
        if (!h || nvec < 0 || (nvec > 0 && (!r_dev || !z_dev))) return fail(PS_EINVAL, "NULL vector");
        if (nvec == 0) return PS_OK;
        h->solver.preconditionBlock(nvec, r_dev, z_dev, cuda_stream);
        return PS_OK;
    });
}

ps_status ps_fea_apply(ps_fea_t* h, int32_t level, const double* x, double* y, int32_t raw) {
    return guarded([&] {
        if (!h || !x || !y) return fail(PS_EINVAL, "NULL vector");
        h->solver.apply(level, x, y, raw != 0);
        return PS_OK;
    });
}

ps_status ps_fea_stresses(ps_fea_t* h, const double* u, double E, double vox, int32_t principals, float* vm, float* p1, float* p3) {
    return guarded([&] {
        if (!h || !u || !vm || (principals && (!p1 || !p3))) return fail(PS_EINVAL, "NULL vector");
        h->solver.stresses(u, E, vox, principals != 0, vm, p1, p3);
        return PS_OK;
    });
}

ps_status ps_fea_reactions(ps_fea_t* h, const double* u, const double* f, double reaction[3]) {
    return guarded([&] {
        if (!h || !u || !reaction) return fail(PS_EINVAL, "NULL vector");
        h->solver.reactions(u, f, reaction);
        return PS_OK;
    });
}

ps_status ps_fea_set_stream(ps_fea_t* h, void* cuda_stream) {
    return guarded([&] {
        if (!h) return fail(PS_EINVAL, "NULL handle");
        h->solver.setStream(cuda_stream);
        return PS_OK;
    });
}

ps_status ps_fea_time_kernel(ps_fea_t* h, int32_t which, int32_t reps, double* ms) {
    return guarded([&] {
        if (!h || !ms || reps < 1 || (which != 0 && which != 1)) return fail(PS_EINVAL, "invalid arguments");
        *ms = h->solver.timeKernel(which, reps);
        return PS_OK;
    });
}

ps_status ps_fea_apply_dot_noalloc(ps_fea_t* h, const double* x_dev, double* y_dev, double* dot_dev, void* cuda_stream) {
    return guarded([&] {
        if (!h || !x_dev || !y_dev || !dot_dev) return fail(PS_EINVAL, "NULL pointer");
        h->solver.applyDotStatic(x_dev, y_dev, dot_dev, cuda_stream);
        return PS_OK;
    });
}

int64_t ps_fea_kernel_launches(const ps_fea_t* h) { return h ? h->solver.launches() : 0; }

int64_t ps_fea_ndof(const ps_fea_t* h) { return h ? h->solver.nDof() : 0; }

int32_t ps_fea_num_levels(const ps_fea_t* h) { return h ? int32_t(h->solver.hierarchy().levels.size()) : 0; }

ps_status ps_fea_level_info(const ps_fea_t* h, int32_t level, int64_t info[9]) {
    if (!h || !info || level < 0 || level >= ps_fea_num_levels(h)) return fail(PS_EINVAL, "level out of range");
    const auto& H = h->solver.hierarchy();
    const auto& L = H.levels[size_t(level)];
    info[0] = L.nx; info[1] = L.ny; info[2] = L.nz; info[3] = L.nNodes; info[4] = L.nDof; info[5] = L.freeDof;
    info[6] = L.nElems; info[7] = L.nOwn; info[8] = H.coarseM;
    return PS_OK;
}

ps_status ps_fea_level_fixed(const ps_fea_t* h, int32_t level, uint8_t* out) {
    if (!h || !out || level < 0 || level >= ps_fea_num_levels(h)) return fail(PS_EINVAL, "level out of range");
    const auto& L = h->solver.hierarchy().levels[size_t(level)];
    for (int64_t n = 0; n < L.nNodes; n++)
        for (int d = 0; d < 3; d++) out[3 * n + d] = (L.nmask[size_t(n)] >> d) & 1;
    return PS_OK;
}

double ps_fea_level_lmax(const ps_fea_t* h, int32_t level) {
    if (!h || level < 0 || level >= ps_fea_num_levels(h)) return 0;
    return h->solver.levelLmax(level);
}

int64_t ps_fea_device_bytes(const ps_fea_t* h) { return h ? h->solver.deviceBytes() : 0; }

ps_status ps_element_matrix(double nu, double K[576], double* corner_stress) {
    return guarded([&] {
        if (!K) return fail(PS_EINVAL, "NULL output");
        const auto el = psfea::hexElement(nu);
        std::memcpy(K, el.K, sizeof el.K);
        if (corner_stress) std::memcpy(corner_stress, el.cornerStress, sizeof el.cornerStress);
        return PS_OK;
    });
}

ps_status ps_prune_floating(const int32_t dims[3], const float* density, const uint8_t* held_node, float* out, int32_t* removed) {
    return guarded([&] {
        if (!dims || !density || !held_node || !out || dims[0] < 1 || dims[1] < 1 || dims[2] < 1)
            return fail(PS_EINVAL, "The structural grid must have three positive dimensions.");
        const int nx = dims[0], ny = dims[1], nz = dims[2];
        const int64_t NX = nx + 1, NY = ny + 1, nE = int64_t(nx) * ny * nz;
        std::vector<uint8_t> seen(size_t(nE), 0);
        std::vector<int64_t> queue;
        for (int64_t e = 0; e < nE; e++) {
            if (!(density[e] > 0)) continue;
            const int i = int(e % nx), j = int((e / nx) % ny), k = int(e / (int64_t(nx) * ny));
            for (int a = 0; a < 8; a++) {
                const int64_t n = (i + psfea::CORNER_XYZ[a][0]) + NX * ((j + psfea::CORNER_XYZ[a][1]) + NY * (k + psfea::CORNER_XYZ[a][2]));
                if (held_node[n]) {
                    seen[size_t(e)] = 1;
                    queue.push_back(e);
                    break;
                }
            }
        }
        for (size_t q = 0; q < queue.size(); q++) {
            const int64_t e = queue[q];
            const int i = int(e % nx), j = int((e / nx) % ny), k = int(e / (int64_t(nx) * ny));
            const int64_t nb[6] = {i > 0 ? e - 1 : -1, i < nx - 1 ? e + 1 : -1, j > 0 ? e - nx : -1, j < ny - 1 ? e + nx : -1,
                                   k > 0 ? e - int64_t(nx) * ny : -1, k < nz - 1 ? e + int64_t(nx) * ny : -1};
            for (int64_t m : nb)
                if (m >= 0 && !seen[size_t(m)] && density[m] > 0) {
                    seen[size_t(m)] = 1;
                    queue.push_back(m);
                }
        }
        int32_t rem = 0;
        for (int64_t e = 0; e < nE; e++) {
            const bool keep = density[e] > 0 && seen[size_t(e)];
            out[e] = keep ? density[e] : 0.f;
            if (density[e] > 0 && !keep) rem++;
        }
        if (removed) *removed = rem;
        return PS_OK;
    });
}

}  // extern "C"

// ---- host-only hierarchy inspection

struct ps_hierarchy {
    psfea::Hierarchy H;
};

extern "C" {

ps_status ps_hierarchy_create(const int32_t dims[3], const float* density, double nu, const uint8_t* bc, int64_t coarsest_max_dof,
                              const double* diag_add, ps_hierarchy_t** out) {
    return guarded([&] {
        if (!out || !dims) return fail(PS_EINVAL, "The structural grid must have three positive dimensions.");
        *out = nullptr;
        auto* h = new ps_hierarchy;
        try {
            h->H = psfea::buildHierarchy(dims, density, nu, bc, coarsest_max_dof, diag_add);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
        return PS_OK;
    });
}

ps_status ps_hierarchy_create_dev(const int32_t dims[3], const float* density, double nu, const uint8_t* bc, int64_t coarsest_max_dof,
                                  const double* diag_add, ps_hierarchy_t** out) {
    return guarded([&] {
        if (!out || !dims) return fail(PS_EINVAL, "The structural grid must have three positive dimensions.");
        *out = nullptr;
        auto engine = psfea::makeDeviceGalerkin();
        auto* h = new ps_hierarchy;
        try {
            h->H = psfea::buildHierarchy(dims, density, nu, bc, coarsest_max_dof, diag_add, engine.get());
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
        return PS_OK;
    });
}

int32_t ps_hierarchy_num_levels(const ps_hierarchy_t* h) { return h ? int32_t(h->H.levels.size()) : 0; }

ps_status ps_hierarchy_level_info(const ps_hierarchy_t* h, int32_t level, int64_t info[9]) {
    if (!h || !info || level < 0 || level >= ps_hierarchy_num_levels(h)) return fail(PS_EINVAL, "level out of range");
    const auto& L = h->H.levels[size_t(level)];
    info[0] = L.nx; info[1] = L.ny; info[2] = L.nz; info[3] = L.nNodes; info[4] = L.nDof; info[5] = L.freeDof;
    info[6] = L.nElems; info[7] = L.nOwn; info[8] = h->H.coarseM;
    return PS_OK;
}

ps_status ps_hierarchy_level_fixed(const ps_hierarchy_t* h, int32_t level, uint8_t* out) {
    if (!h || !out || level < 0 || level >= ps_hierarchy_num_levels(h)) return fail(PS_EINVAL, "level out of range");
    const auto& L = h->H.levels[size_t(level)];
    for (int64_t n = 0; n < L.nNodes; n++)
        for (int d = 0; d < 3; d++) out[3 * n + d] = (L.nmask[size_t(n)] >> d) & 1;
    return PS_OK;
}

ps_status ps_hierarchy_level_own(const ps_hierarchy_t* h, int32_t level, float* out) {
    if (!h || !out || level < 0 || level >= ps_hierarchy_num_levels(h)) return fail(PS_EINVAL, "level out of range");
    const auto& L = h->H.levels[size_t(level)];
    if (!L.own.empty()) std::memcpy(out, L.own.data(), L.own.size() * sizeof(float));
    return PS_OK;
}

ps_status ps_hierarchy_level_kb(const ps_hierarchy_t* h, int32_t level, double* out) {
    if (!h || !out || level < 0 || level >= ps_hierarchy_num_levels(h)) return fail(PS_EINVAL, "level out of range");
    std::memcpy(out, h->H.levels[size_t(level)].Kb, 576 * sizeof(double));
    return PS_OK;
}

void ps_hierarchy_destroy(ps_hierarchy_t* h) { delete h; }

}  // extern "C"
