// ORACLE — test infrastructure only. A plain CPU restatement of Parts Sim's linear-static voxel
// solve (native/src/fea/hex8.cpp and native/src/fea/voxel_fea.cpp), used by tests/, the smoke
// check and bench.py's CPU-baseline leg as the checker. Nothing in the product links or calls it.
//
// Parity is pinned two ways: against golden vectors written by the reference itself
// (tests/golden/, generated by tests/golden/make_golden.py from the reference compiled into
// oracle/_ref), and, where oracle/_ref is present, against the reference run side by side.
//
// Deliberately simple: scalar loops, element-by-element gathers (no assembled stencil), so its
// rounding differs from the reference's in the last bits but its mathematics is the same.
// Every function names the reference lines it follows.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <functional>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace orc {

using std::int64_t;

// corner a of a voxel sits at unit offset CORNER[a] (hex8.hpp:14: bottom face CCW, then top face)
static const int CORNER[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
static int cornerOf(int x, int y, int z) {
    for (int a = 0; a < 8; a++)
        if (CORNER[a][0] == x && CORNER[a][1] == y && CORNER[a][2] == z) return a;
    return -1;
}

// ---- parallel helper (oracle speed only; results do not depend on it: no reductions) ----
static void parFor(int64_t n, const std::function<void(int64_t, int64_t)>& fn) {
    unsigned T = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    if (n < 4096 || T == 1) { fn(0, n); return; }
    std::vector<std::thread> th;
    for (unsigned t = 0; t < T; t++) {
        int64_t a = n * t / T, b = n * (t + 1) / T;
        th.emplace_back([=, &fn] { if (a < b) fn(a, b); });
    }
    for (auto& x : th) x.join();
}

// ---- element (hex8.cpp:8-155) ----

// isotropic D for E = 1, Voigt order xx yy zz xy yz zx (hex8.cpp:8-18)
static void elasticity(double nu, double D[36]) {
    if (!std::isfinite(nu) || nu <= -1 || nu >= 0.5) throw std::invalid_argument("Poisson's ratio must be greater than -1 and less than 0.5.");
    const double lam = nu / ((1 + nu) * (1 - 2 * nu)), mu = 1 / (2 * (1 + nu));
    for (int i = 0; i < 36; i++) D[i] = 0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) D[i * 6 + j] = lam + (i == j ? 2 * mu : 0);
    for (int i = 3; i < 6; i++) D[i * 6 + i] = mu;
}

// strain rows of one displacement triple with shape gradient g (hex8.cpp:20-30)
static void strainCols(double* B, int ncol, int c, double gx, double gy, double gz) {
    B[0 * ncol + c] = gx;
    B[1 * ncol + c + 1] = gy;
    B[2 * ncol + c + 2] = gz;
    B[3 * ncol + c] = gy;
    B[3 * ncol + c + 1] = gx;
    B[4 * ncol + c + 1] = gz;
    B[4 * ncol + c + 2] = gy;
    B[5 * ncol + c] = gz;
    B[5 * ncol + c + 2] = gx;
}

// B (6x24) at natural point (xi, eta, zeta) on the unit cube (hex8.cpp:32-43)
static void bmatrix(double xi, double eta, double zeta, double B[144]) {
    for (int i = 0; i < 144; i++) B[i] = 0;
    for (int a = 0; a < 8; a++) {
        const double sx = 2.0 * CORNER[a][0] - 1, sy = 2.0 * CORNER[a][1] - 1, sz = 2.0 * CORNER[a][2] - 1;
        // dN/dx = dN/dxi * 2 on a unit cube, N = (1 + sx xi)(1 + sy eta)(1 + sz zeta) / 8
        strainCols(B, 24, 3 * a, sx * (1 + sy * eta) * (1 + sz * zeta) / 4, sy * (1 + sx * xi) * (1 + sz * zeta) / 4,
                   sz * (1 + sx * xi) * (1 + sy * eta) / 4);
    }
}

// Wilson bubble-mode strains G (6x9) (hex8.cpp:46-51)
static void bubbles(double xi, double eta, double zeta, double G[54]) {
    for (int i = 0; i < 54; i++) G[i] = 0;
    strainCols(G, 9, 0, -4 * xi, 0, 0);
    strainCols(G, 9, 3, 0, -4 * eta, 0);
    strainCols(G, 9, 6, 0, 0, -4 * zeta);
}

// solve the 9x9 system by Gaussian elimination with partial pivoting: X = A^-1 Bm (9 x n)
static void solve9(std::vector<double> A, std::vector<double>& Bm, int n) {
    for (int c = 0; c < 9; c++) {
        int p = c;
        for (int r = c + 1; r < 9; r++)
            if (std::fabs(A[r * 9 + c]) > std::fabs(A[p * 9 + c])) p = r;
        if (p != c) {
            for (int j = 0; j < 9; j++) std::swap(A[c * 9 + j], A[p * 9 + j]);
            for (int j = 0; j < n; j++) std::swap(Bm[c * n + j], Bm[p * n + j]);
        }
        for (int r = c + 1; r < 9; r++) {
            const double f = A[r * 9 + c] / A[c * 9 + c];
            if (f == 0) continue;
            for (int j = c; j < 9; j++) A[r * 9 + j] -= f * A[c * 9 + j];
            for (int j = 0; j < n; j++) Bm[r * n + j] -= f * Bm[c * n + j];
        }
    }
    for (int c = 8; c >= 0; c--) {
        for (int j = 0; j < n; j++) {
            double s = Bm[c * n + j];
            for (int k = c + 1; k < 9; k++) s -= A[c * 9 + k] * Bm[k * n + j];
            Bm[c * n + j] = s / A[c * 9 + c];
        }
    }
}

struct Element {
    double K[576];
    double cornerStress[8][144];
    double gaussB[8][144];
};

// condensed 24x24 stiffness on the unit cube with E = 1 (hex8.cpp:104-155): 2x2x2 Gauss, the 9
// bubble modes eliminated statically, then symmetrised; corner stress = D Bbar at each corner
static Element element(double nu, bool modes) {
    double D[36];
    elasticity(nu, D);
    const double g = 1 / std::sqrt(3.0), w = 1.0 / 8;  // detJ of the unit cube in natural coordinates
    std::vector<double> Kuu(576, 0.0), Kua(24 * 9, 0.0), Kaa(81, 0.0);
    double B[144], G[54], DB[144], DG[54];
    for (int q = 0; q < 8; q++) {
        const double xi = (CORNER[q][0] ? g : -g), eta = (CORNER[q][1] ? g : -g), ze = (CORNER[q][2] ? g : -g);
        bmatrix(xi, eta, ze, B);
        bubbles(xi, eta, ze, G);
        for (int r = 0; r < 6; r++)
            for (int c = 0; c < 24; c++) {
                double s = 0;
                for (int k = 0; k < 6; k++) s += D[r * 6 + k] * B[k * 24 + c];
                DB[r * 24 + c] = s;
            }
        for (int r = 0; r < 6; r++)
            for (int c = 0; c < 9; c++) {
                double s = 0;
                for (int k = 0; k < 6; k++) s += D[r * 6 + k] * G[k * 9 + c];
                DG[r * 9 + c] = s;
            }
        for (int i = 0; i < 24; i++)
            for (int j = 0; j < 24; j++) {
                double s = 0;
                for (int k = 0; k < 6; k++) s += B[k * 24 + i] * DB[k * 24 + j];
                Kuu[i * 24 + j] += w * s;
            }
        for (int i = 0; i < 24; i++)
            for (int j = 0; j < 9; j++) {
                double s = 0;
                for (int k = 0; k < 6; k++) s += B[k * 24 + i] * DG[k * 9 + j];
                Kua[i * 9 + j] += w * s;
            }
        for (int i = 0; i < 9; i++)
            for (int j = 0; j < 9; j++) {
                double s = 0;
                for (int k = 0; k < 6; k++) s += G[k * 9 + i] * DG[k * 9 + j];
                Kaa[i * 9 + j] += w * s;
            }
    }
    // alpha = Acond u with Acond = -Kaa^-1 Kau (9 x 24)
    std::vector<double> Acond;
    if (modes) {
        Acond.assign(9 * 24, 0.0);
        for (int q = 0; q < 9; q++)
            for (int i = 0; i < 24; i++) Acond[q * 24 + i] = Kua[i * 9 + q];
        solve9(Kaa, Acond, 24);
        for (auto& v : Acond) v = -v;
        for (int i = 0; i < 24; i++)
            for (int j = 0; j < 24; j++) {
                double s = 0;
                for (int q = 0; q < 9; q++) s += Kua[i * 9 + q] * Acond[q * 24 + j];
                Kuu[i * 24 + j] += s;
            }
        for (int i = 0; i < 24; i++)
            for (int j = i + 1; j < 24; j++) Kuu[i * 24 + j] = Kuu[j * 24 + i] = 0.5 * (Kuu[i * 24 + j] + Kuu[j * 24 + i]);
    }
    Element el;
    for (int i = 0; i < 576; i++) el.K[i] = Kuu[i];
    auto enhanced = [&](double xi, double eta, double ze, double out[144]) {
        bmatrix(xi, eta, ze, out);
        if (modes) {
            double Gm[54];
            bubbles(xi, eta, ze, Gm);
            for (int r = 0; r < 6; r++)
                for (int c = 0; c < 24; c++) {
                    double s = 0;
                    for (int q = 0; q < 9; q++) s += Gm[r * 9 + q] * Acond[q * 24 + c];
                    out[r * 24 + c] += s;
                }
        }
    };
    for (int a = 0; a < 8; a++) {
        double Bt[144];
        enhanced(2.0 * CORNER[a][0] - 1, 2.0 * CORNER[a][1] - 1, 2.0 * CORNER[a][2] - 1, Bt);
        for (int r = 0; r < 6; r++)
            for (int c = 0; c < 24; c++) {
                double s = 0;
                for (int k = 0; k < 6; k++) s += D[r * 6 + k] * Bt[k * 24 + c];
                el.cornerStress[a][r * 24 + c] = s;
            }
        enhanced((2.0 * CORNER[a][0] - 1) * g, (2.0 * CORNER[a][1] - 1) * g, (2.0 * CORNER[a][2] - 1) * g, el.gaussB[a]);
    }
    return el;
}

// ---- hierarchy (voxel_fea.cpp:113-386) ----

struct Level {
    int nx = 0, ny = 0, nz = 0, NX = 0, NY = 0, NZ = 0;
    int64_t nNodes = 0, nDof = 0;
    std::vector<int> elems;            // voxel index per element, increasing
    std::vector<int> emap;             // voxel -> element or -1
    std::vector<double> rho;           // scale of elements that are rho * Kb
    std::vector<int> kIdx;             // element -> own matrix or -1 (coarse levels)
    std::vector<float> own;            // own matrices, 576 floats each
    std::vector<std::vector<int>> children;  // coarse element -> fine elements
    std::vector<uint8_t> child;        // fine element -> its child position in its coarse element
    double Kb[576];
    std::vector<uint8_t> bc, fixed, active;
    std::vector<double> diag, invDiag, diagAdd;
    int64_t freeDof = 0;
    double lmax = 0, omega = 0.5;
    std::vector<float> r, z, t, d;
    bool scaled(int e) const { return kIdx.empty() || kIdx[e] < 0; }
    int64_t node(int i, int j, int k) const { return i + int64_t(NX) * (j + int64_t(NY) * k); }
};

static Level makeGrid(int nx, int ny, int nz) {
    Level L;
    L.nx = nx; L.ny = ny; L.nz = nz;
    L.NX = nx + 1; L.NY = ny + 1; L.NZ = nz + 1;
    L.nNodes = int64_t(L.NX) * L.NY * L.NZ;
    L.nDof = 3 * L.nNodes;
    return L;
}

// element matrix entry (r, c) of element e, as a double
static inline double kEntry(const Level& L, int e, int r, int c) {
    return L.scaled(e) ? L.rho[e] * L.Kb[r * 24 + c] : double(L.own[int64_t(L.kIdx[e]) * 576 + r * 24 + c]);
}

// node of element e at corner a
static inline int64_t cornerNode(const Level& L, int e, int a) {
    const int v = L.elems[e];
    const int i = v % L.nx, j = (v / L.nx) % L.ny, k = v / (L.nx * L.ny);
    return L.node(i + CORNER[a][0], j + CORNER[a][1], k + CORNER[a][2]);
}

// diagonal, fixed mask, free count (voxel_fea.cpp:208-234)
static void finish(Level& L) {
    L.active.assign(L.nNodes, 0);
    L.diag.assign(L.nDof, 0.0);
    for (int e = 0; e < int(L.elems.size()); e++)
        for (int a = 0; a < 8; a++) {
            const int64_t n = cornerNode(L, e, a);
            L.active[n] = 1;
            for (int d = 0; d < 3; d++) L.diag[3 * n + d] += kEntry(L, e, 3 * a + d, 3 * a + d);
        }
    if (!L.diagAdd.empty())
        for (int64_t i = 0; i < L.nDof; i++) L.diag[i] += L.diagAdd[i];
    L.fixed.assign(L.nDof, 0);
    L.invDiag.assign(L.nDof, 0.0);
    L.freeDof = 0;
    for (int64_t n = 0; n < L.nNodes; n++)
        for (int d = 0; d < 3; d++) {
            const int64_t i = 3 * n + d;
            if (!L.active[n] || L.bc[i] || !(L.diag[i] > 0)) L.fixed[i] = 1;
            else { L.invDiag[i] = 1 / L.diag[i]; L.freeDof++; }
        }
    L.r.assign(L.nDof, 0.f);
    L.z.assign(L.nDof, 0.f);
    L.t.assign(L.nDof, 0.f);
    L.d.assign(L.nDof, 0.f);
}

// interpolation weights of coarse corner b at the fine child c's corner a (voxel_fea.cpp:61-83)
static double childWeight(int c, int a, int b) {
    const double s[3] = {((c & 1) + CORNER[a][0]) / 2.0, (((c >> 1) & 1) + CORNER[a][1]) / 2.0, (((c >> 2) & 1) + CORNER[a][2]) / 2.0};
    double w = 1;
    for (int d = 0; d < 3; d++) w *= CORNER[b][d] ? s[d] : 1 - s[d];
    return w;
}

// dense 24x24 prolongation of child c: P[3a + d][3b + d] = w(c, a, b)
static void childP(int c, double P[576]) {
    for (int i = 0; i < 576; i++) P[i] = 0;
    for (int a = 0; a < 8; a++)
        for (int b = 0; b < 8; b++) {
            const double w = childWeight(c, a, b);
            if (w > 1e-12)
                for (int d = 0; d < 3; d++) P[(3 * a + d) * 24 + 3 * b + d] = w;
        }
}

// out += s * P^T K P (voxel_fea.cpp:86-111, as a plain triple product)
static void galerkin(double* out, const double* K, const double* P, double s) {
    double KP[576];
    for (int i = 0; i < 24; i++)
        for (int j = 0; j < 24; j++) {
            double acc = 0;
            for (int k = 0; k < 24; k++) acc += K[i * 24 + k] * P[k * 24 + j];
            KP[i * 24 + j] = acc;
        }
    for (int i = 0; i < 24; i++)
        for (int j = 0; j < 24; j++) {
            double acc = 0;
            for (int k = 0; k < 24; k++) acc += P[k * 24 + i] * KP[k * 24 + j];
            out[i * 24 + j] += s * acc;
        }
}

// restriction P^T v, coarse node I gathers fine 2I (weight 1) and 2I +- 1 (weight 1/2) per axis
// (voxel_fea.cpp:739-779)
template <class T>
static void restrictTo(const Level& F, const Level& C, const T* rf, T* rc, bool zeroFixed) {
    parFor(C.nNodes, [&](int64_t lo, int64_t hi) {
        for (int64_t cn = lo; cn < hi; cn++) {
            const int I = int(cn % C.NX), J = int((cn / C.NX) % C.NY), K = int(cn / (int64_t(C.NX) * C.NY));
            T s[3] = {0, 0, 0};
            for (int dk = -1; dk <= 1; dk++)
                for (int dj = -1; dj <= 1; dj++)
                    for (int di = -1; di <= 1; di++) {
                        const int i = 2 * I + di, j = 2 * J + dj, k = 2 * K + dk;
                        if (i < 0 || j < 0 || k < 0 || i >= F.NX || j >= F.NY || k >= F.NZ) continue;
                        const T w = T(di ? 0.5 : 1) * T(dj ? 0.5 : 1) * T(dk ? 0.5 : 1);
                        const T* p = rf + 3 * F.node(i, j, k);
                        for (int d = 0; d < 3; d++) s[d] += w * p[d];
                    }
            for (int d = 0; d < 3; d++) rc[3 * cn + d] = (zeroFixed && (C.fixed[3 * cn + d] || !C.active[cn])) ? T(0) : s[d];
        }
    });
}

// trilinear prolongation added into free fine DOFs (voxel_fea.cpp:781-815)
template <class T>
static void prolongAdd(const Level& F, const Level& C, const T* zc, T* zf) {
    parFor(F.nNodes, [&](int64_t lo, int64_t hi) {
        for (int64_t fn = lo; fn < hi; fn++) {
            if (!F.active[fn]) continue;
            const int i = int(fn % F.NX), j = int((fn / F.NX) % F.NY), k = int(fn / (int64_t(F.NX) * F.NY));
            T s[3] = {0, 0, 0};
            const int is[2] = {i / 2, (i & 1) ? i / 2 + 1 : -1}, js[2] = {j / 2, (j & 1) ? j / 2 + 1 : -1}, ks[2] = {k / 2, (k & 1) ? k / 2 + 1 : -1};
            const T w = T((i & 1) ? 0.5 : 1) * T((j & 1) ? 0.5 : 1) * T((k & 1) ? 0.5 : 1);
            for (int a = 0; a < 2; a++)
                for (int b = 0; b < 2; b++)
                    for (int c = 0; c < 2; c++) {
                        if (is[a] < 0 || js[b] < 0 || ks[c] < 0) continue;
                        const T* p = zc + 3 * C.node(is[a], js[b], ks[c]);
                        for (int d = 0; d < 3; d++) s[d] += w * p[d];
                    }
            for (int d = 0; d < 3; d++)
                if (!F.fixed[3 * fn + d]) zf[3 * fn + d] += s[d];
        }
    });
}

// next coarser level with exact Galerkin elements (voxel_fea.cpp:268-386)
static Level coarsen(Level& F) {
    Level C = makeGrid((F.nx + 1) / 2, (F.ny + 1) / 2, (F.nz + 1) / 2);
    const int64_t nCv = int64_t(C.nx) * C.ny * C.nz;
    C.emap.assign(nCv, -1);
    std::vector<uint8_t> used(nCv, 0);
    F.child.assign(F.elems.size(), 0);
    for (int e = 0; e < int(F.elems.size()); e++) {
        const int v = F.elems[e], i = v % F.nx, j = (v / F.nx) % F.ny, k = v / (F.nx * F.ny);
        used[(i / 2) + int64_t(C.nx) * ((j / 2) + int64_t(C.ny) * (k / 2))] = 1;
        F.child[e] = uint8_t((i & 1) | ((j & 1) << 1) | ((k & 1) << 2));
    }
    for (int64_t v = 0; v < nCv; v++)
        if (used[v]) { C.emap[v] = int(C.elems.size()); C.elems.push_back(int(v)); }
    C.children.assign(C.elems.size(), {});
    for (int e = 0; e < int(F.elems.size()); e++) {
        const int v = F.elems[e], i = v % F.nx, j = (v / F.nx) % F.ny, k = v / (F.nx * F.ny);
        C.children[C.emap[(i / 2) + int64_t(C.nx) * ((j / 2) + int64_t(C.ny) * (k / 2))]].push_back(e);
    }
    // uniform element: sum over the 8 child positions of P_c^T Kb P_c
    double P[8][576];
    for (int c = 0; c < 8; c++) childP(c, P[c]);
    double Kc[576] = {0};
    for (int c = 0; c < 8; c++) galerkin(Kc, F.Kb, P[c], 1.0);
    std::memcpy(C.Kb, Kc, sizeof Kc);
    const int nE = int(C.elems.size());
    C.rho.assign(nE, 0.0);
    C.kIdx.assign(nE, -1);
    int nOwn = 0;
    for (int q = 0; q < nE; q++) {
        const auto& ch = C.children[q];
        bool uniform = ch.size() == 8 && F.scaled(ch[0]);
        const double s = uniform ? F.rho[ch[0]] : 0;
        for (int f : ch) uniform = uniform && F.scaled(f) && F.rho[f] == s;
        if (uniform) C.rho[q] = s;
        else C.kIdx[q] = nOwn++;
    }
    C.own.assign(int64_t(nOwn) * 576, 0.f);
    parFor(nE, [&](int64_t lo, int64_t hi) {
        std::vector<double> out(576), Kf(576);
        for (int64_t q = lo; q < hi; q++) {
            if (C.kIdx[q] < 0) continue;
            std::fill(out.begin(), out.end(), 0.0);
            for (int f : C.children[q]) {
                for (int u = 0; u < 576; u++) Kf[u] = F.scaled(f) ? F.Kb[u] : double(F.own[int64_t(F.kIdx[f]) * 576 + u]);
                galerkin(out.data(), Kf.data(), P[F.child[f]], F.scaled(f) ? F.rho[f] : 1.0);
            }
            for (int u = 0; u < 576; u++) C.own[int64_t(C.kIdx[q]) * 576 + u] = float(out[u]);
        }
    });
    // held coarse DOF: OR over the fine DOFs it interpolates to (voxel_fea.cpp:355-378)
    C.bc.assign(C.nDof, 0);
    for (int k = 0; k < F.NZ; k++)
        for (int j = 0; j < F.NY; j++)
            for (int i = 0; i < F.NX; i++) {
                const int64_t fn = F.node(i, j, k);
                for (int kk = k / 2; kk <= (k + 1) / 2; kk++)
                    for (int jj = j / 2; jj <= (j + 1) / 2; jj++)
                        for (int ii = i / 2; ii <= (i + 1) / 2; ii++) {
                            const int64_t cn = C.node(ii, jj, kk);
                            for (int d = 0; d < 3; d++) C.bc[3 * cn + d] |= F.bc[3 * fn + d];
                        }
            }
    if (!F.diagAdd.empty()) {
        C.diagAdd.assign(C.nDof, 0.0);
        restrictTo<double>(F, C, F.diagAdd.data(), C.diagAdd.data(), false);
    }
    finish(C);
    return C;
}

// ---- operator, smoother, V-cycle, CG (voxel_fea.cpp:393-927) ----

struct Model {
    double nu;
    Element el;
    std::vector<Level> levels;
    std::vector<int64_t> cmap;  // coarsest DOF -> dense index or -1
    int64_t m = 0;
    std::vector<double> chol;   // lower Cholesky factor, row-major m x m

    // y = K x on level l, held/inactive DOFs zeroed unless raw (voxel_fea.cpp:393-504):
    // every node gathers the rows of its corner in each of its (up to 8) voxels
    template <class T>
    void apply(int l, const T* x, T* y, bool raw) const {
        const Level& L = levels[l];
        parFor(L.nNodes, [&](int64_t lo, int64_t hi) {
            for (int64_t n = lo; n < hi; n++) {
                const int i = int(n % L.NX), j = int((n / L.NX) % L.NY), k = int(n / (int64_t(L.NX) * L.NY));
                T acc[3] = {0, 0, 0};
                if (L.active[n]) {
                    for (int v = 0; v < 8; v++) {
                        const int di = v & 1, dj = (v >> 1) & 1, dk = v >> 2;
                        const int ei = i - 1 + di, ej = j - 1 + dj, ek = k - 1 + dk;
                        if (ei < 0 || ej < 0 || ek < 0 || ei >= L.nx || ej >= L.ny || ek >= L.nz) continue;
                        const int e = L.emap[ei + int64_t(L.nx) * (ej + int64_t(L.ny) * ek)];
                        if (e < 0) continue;
                        const int a = cornerOf(1 - di, 1 - dj, 1 - dk);
                        for (int b = 0; b < 8; b++) {
                            const T* xb = x + 3 * L.node(ei + CORNER[b][0], ej + CORNER[b][1], ek + CORNER[b][2]);
                            for (int d = 0; d < 3; d++)
                                for (int c = 0; c < 3; c++) {
                                    const T kv = L.scaled(e) ? T(L.rho[e]) * T(L.Kb[(3 * a + d) * 24 + 3 * b + c])
                                                             : T(L.own[int64_t(L.kIdx[e]) * 576 + (3 * a + d) * 24 + 3 * b + c]);
                                    acc[d] += kv * xb[c];
                                }
                        }
                    }
                    if (!L.diagAdd.empty())
                        for (int d = 0; d < 3; d++) acc[d] += T(L.diagAdd[3 * n + d]) * x[3 * n + d];
                }
                for (int d = 0; d < 3; d++) y[3 * n + d] = (!raw && L.fixed[3 * n + d]) ? T(0) : acc[d];
            }
        });
    }

    // largest eigenvalue of a symmetric tridiagonal matrix by bisection on Sturm counts (voxel_fea.cpp:506-530)
    static double tridiagMax(const std::vector<double>& a, const std::vector<double>& b) {
        const int k = int(a.size());
        double lo = INFINITY, hi = -INFINITY;
        for (int i = 0; i < k; i++) {
            const double r = (i > 0 ? std::fabs(b[i - 1]) : 0) + (i + 1 < k ? std::fabs(b[i]) : 0);
            lo = std::min(lo, a[i] - r);
            hi = std::max(hi, a[i] + r);
        }
        for (int it = 0; it < 100 && hi - lo > 1e-12 * std::fabs(hi); it++) {
            const double mid = 0.5 * (lo + hi);
            int count = 0;
            double q = 1;
            for (int i = 0; i < k; i++) {
                q = a[i] - mid - (i > 0 ? b[i - 1] * b[i - 1] / q : 0);
                if (q == 0) q = 1e-300;
                if (q > 0) count++;
            }
            if (count > 0) lo = mid;
            else hi = mid;
        }
        return hi;
    }

    // 10 Lanczos steps on D^-1/2 K D^-1/2 from the LCG start vector (voxel_fea.cpp:579-610)
    void lanczos(int l) {
        Level& L = levels[l];
        const int64_t n = L.nDof;
        std::vector<double> sq(n), v(n), vp(n, 0.0), w(n), x(n);
        for (int64_t i = 0; i < n; i++) sq[i] = std::sqrt(L.invDiag[i]);
        uint32_t seed = 12345;
        double nv = 0;
        for (int64_t i = 0; i < n; i++) {
            seed = (seed * 1103515245u + 12345u) & 0x7fffffffu;
            v[i] = L.fixed[i] ? 0 : double(seed) / 0x7fffffff - 0.5;
        }
        for (int64_t i = 0; i < n; i++) nv += v[i] * v[i];
        nv = std::sqrt(nv);
        for (auto& e : v) e /= nv > 0 ? nv : 1;
        std::vector<double> al, be;
        double b = 0;
        for (int s = 0; s < 10; s++) {
            for (int64_t i = 0; i < n; i++) x[i] = sq[i] * v[i];
            apply<double>(l, x.data(), w.data(), false);
            for (int64_t i = 0; i < n; i++) w[i] = sq[i] * w[i] - b * vp[i];
            double a = 0;
            for (int64_t i = 0; i < n; i++) a += w[i] * v[i];
            for (int64_t i = 0; i < n; i++) w[i] -= a * v[i];
            al.push_back(a);
            double bb = 0;
            for (int64_t i = 0; i < n; i++) bb += w[i] * w[i];
            b = std::sqrt(bb);
            if (!(b > 1e-12 * std::fabs(a))) break;
            be.push_back(b);
            std::swap(vp, v);
            for (int64_t i = 0; i < n; i++) v[i] = w[i] / b;
        }
        be.resize(al.size() - 1);
        L.lmax = tridiagMax(al, be);
        L.omega = 1.2 / (L.lmax * 1.05);
    }

    void prepare() {
        for (int l = 0; l + 1 < int(levels.size()); l++)
            if (!(levels[l].lmax > 0)) lanczos(l);
    }

    // dense coarsest matrix and its Cholesky factor with the tiny-pivot rule (voxel_fea.cpp:612-661)
    void factorCoarsest() {
        const Level& L = levels.back();
        cmap.assign(L.nDof, -1);
        m = 0;
        for (int64_t i = 0; i < L.nDof; i++)
            if (!L.fixed[i]) cmap[i] = m++;
        chol.clear();
        if (m == 0 || m > 3000) return;
        std::vector<double>& A = chol;
        A.assign(m * m, 0.0);
        for (int e = 0; e < int(L.elems.size()); e++) {
            int64_t dofs[24];
            for (int a = 0; a < 8; a++)
                for (int d = 0; d < 3; d++) dofs[3 * a + d] = cmap[3 * cornerNode(L, e, a) + d];
            for (int r = 0; r < 24; r++)
                for (int c = 0; c < 24; c++)
                    if (dofs[r] >= 0 && dofs[c] >= 0) A[dofs[r] * m + dofs[c]] += kEntry(L, e, r, c);
        }
        if (!L.diagAdd.empty())
            for (int64_t i = 0; i < L.nDof; i++)
                if (cmap[i] >= 0) A[cmap[i] * m + cmap[i]] += L.diagAdd[i];
        double maxDiag = 0;
        for (int64_t i = 0; i < m; i++) maxDiag = std::max(maxDiag, A[i * m + i]);
        for (int64_t j = 0; j < m; j++) {
            double s = A[j * m + j];
            for (int64_t k = 0; k < j; k++) s -= A[j * m + k] * A[j * m + k];
            // the reference's right-looking update leaves A[j][j] minus the same squares here
            if (!(s > 1e-10 * maxDiag)) s = maxDiag;
            const double ljj = std::sqrt(s);
            A[j * m + j] = ljj;
            for (int64_t i = j + 1; i < m; i++) {
                double t = A[i * m + j];
                for (int64_t k = 0; k < j; k++) t -= A[i * m + k] * A[j * m + k];
                A[i * m + j] = t / ljj;
            }
        }
        for (int64_t i = 0; i < m; i++)
            for (int64_t j = i + 1; j < m; j++) A[i * m + j] = 0;
    }

    // L L^T y = b (dense.hpp:26-34)
    void cholSolve(double* y) const {
        for (int64_t i = 0; i < m; i++) {
            double s = y[i];
            for (int64_t k = 0; k < i; k++) s -= chol[i * m + k] * y[k];
            y[i] = s / chol[i * m + i];
        }
        for (int64_t i = m - 1; i >= 0; i--) {
            double s = y[i];
            for (int64_t k = i + 1; k < m; k++) s -= chol[k * m + i] * y[k];
            y[i] = s / chol[i * m + i];
        }
    }

    // degree-2 Chebyshev on [0.1, 1.15] lmax (voxel_fea.cpp:692-725)
    static void chebCoefs(double lmax, double& c0, double& c1, double& c2) {
        const double b = 1.15 * lmax, a = 0.1 * lmax;
        const double theta = (b + a) / 2, delta = (b - a) / 2, sigma = theta / delta;
        const double rho0 = 1 / sigma, rho1 = 1 / (2 * sigma - rho0);
        c0 = 1 / theta;
        c1 = rho1 * rho0;
        c2 = 2 * rho1 / delta;
    }

    void chebyshev(int l, bool first) {
        Level& L = levels[l];
        double cc0, cc1, cc2;
        chebCoefs(L.lmax, cc0, cc1, cc2);
        const float c0 = float(cc0), c1 = float(cc1), c2 = float(cc2);
        const int64_t n = L.nDof;
        std::vector<float> D(n);
        for (int64_t i = 0; i < n; i++) D[i] = float(L.invDiag[i]);
        if (first) {
            for (int64_t i = 0; i < n; i++) { L.d[i] = c0 * D[i] * L.r[i]; L.z[i] = L.d[i]; }
        } else {
            apply<float>(l, L.z.data(), L.t.data(), false);
            for (int64_t i = 0; i < n; i++) { L.d[i] = c0 * D[i] * (L.r[i] - L.t[i]); L.z[i] += L.d[i]; }
        }
        apply<float>(l, L.z.data(), L.t.data(), false);
        for (int64_t i = 0; i < n; i++) { L.d[i] = c1 * L.d[i] + c2 * D[i] * (L.r[i] - L.t[i]); L.z[i] += L.d[i]; }
    }

    void jacobi(int l, bool first) {
        Level& L = levels[l];
        const float om = float(L.omega);
        if (first) {
            for (int64_t i = 0; i < L.nDof; i++) L.z[i] = om * float(L.invDiag[i]) * L.r[i];
            return;
        }
        apply<float>(l, L.z.data(), L.t.data(), false);
        for (int64_t i = 0; i < L.nDof; i++) L.z[i] += om * float(L.invDiag[i]) * (L.r[i] - L.t[i]);
    }

    void coarseSolve() {
        Level& L = levels.back();
        std::fill(L.z.begin(), L.z.end(), 0.f);
        if (chol.empty()) {
            for (int s = 0; s < 40; s++) jacobi(int(levels.size()) - 1, s == 0);
            return;
        }
        std::vector<double> y(m);
        for (int64_t i = 0; i < L.nDof; i++)
            if (cmap[i] >= 0) y[cmap[i]] = L.r[i];
        cholSolve(y.data());
        for (int64_t i = 0; i < L.nDof; i++)
            if (cmap[i] >= 0) L.z[i] = float(y[cmap[i]]);
    }

    // (voxel_fea.cpp:817-828)
    void vcycle(int l) {
        Level& L = levels[l];
        if (l == int(levels.size()) - 1) { coarseSolve(); return; }
        Level& C = levels[l + 1];
        chebyshev(l, true);
        apply<float>(l, L.z.data(), L.t.data(), false);
        for (int64_t i = 0; i < L.nDof; i++) L.t[i] = L.fixed[i] ? 0.f : L.r[i] - L.t[i];
        restrictTo<float>(L, C, L.t.data(), C.r.data(), true);
        vcycle(l + 1);
        prolongAdd<float>(L, C, C.z.data(), L.z.data());
        chebyshev(l, false);
    }

    // one V-cycle in 32-bit with r scaled to order one (voxel_fea.cpp:835-861)
    void precondition(const double* r, double* z) {
        Level& L = levels[0];
        const int64_t n = L.nDof;
        if (levels.size() == 1 && !chol.empty()) {
            std::vector<double> y(m);
            for (int64_t i = 0; i < n; i++)
                if (cmap[i] >= 0) y[cmap[i]] = r[i];
            cholSolve(y.data());
            for (int64_t i = 0; i < n; i++) z[i] = cmap[i] >= 0 ? y[cmap[i]] : 0;
            return;
        }
        double rmax = 0;
        for (int64_t i = 0; i < n; i++)
            if (!L.fixed[i]) rmax = std::max(rmax, std::fabs(r[i]));
        if (!(rmax > 0)) { std::fill(z, z + n, 0.0); return; }
        const double s = 1 / rmax;
        for (int64_t i = 0; i < n; i++) L.r[i] = L.fixed[i] ? 0.f : float(r[i] * s);
        vcycle(0);
        for (int64_t i = 0; i < n; i++) z[i] = L.active[i / 3] ? double(L.z[i]) * rmax : 0.0;
    }

    struct Result { int iterations = 0; double residual = 0; bool converged = false; };

    // flexible PCG with Polak-Ribiere beta, true residual reported (voxel_fea.cpp:863-927)
    Result solve(const double* f, double tol, int maxIter, const double* x0, double* x) {
        Level& L = levels[0];
        const int64_t n = L.nDof;
        for (int64_t i = 0; i < n; i++)
            if (!std::isfinite(f[i]) || (x0 && !std::isfinite(x0[i]))) throw std::invalid_argument("Forces and displacements must be finite numbers.");
        Result res;
        for (int64_t i = 0; i < n; i++) x[i] = (x0 && !L.fixed[i]) ? x0[i] : 0.0;
        double bnorm = 0;
        for (int64_t i = 0; i < n; i++)
            if (!L.fixed[i]) bnorm += f[i] * f[i];
        bnorm = std::sqrt(bnorm);
        if (bnorm == 0) {
            std::fill(x, x + n, 0.0);
            res.converged = true;
            return res;
        }
        std::vector<double> r(n), p(n), q(n), z(n);
        auto dot = [&](const std::vector<double>& a, const std::vector<double>& b) {
            double s = 0;
            for (int64_t i = 0; i < n; i++) s += a[i] * b[i];
            return s;
        };
        apply<double>(0, x, q.data(), false);
        for (int64_t i = 0; i < n; i++) r[i] = L.fixed[i] ? 0 : f[i] - q[i];
        prepare();
        precondition(r.data(), z.data());
        p = z;
        double rz = dot(r, z);
        double rel = std::sqrt(dot(r, r)) / bnorm;
        int it = 0;
        for (; it < maxIter && rel > tol; it++) {
            apply<double>(0, p.data(), q.data(), false);
            const double pq = dot(p, q);
            if (!(pq > 0)) break;
            const double alpha = rz / pq;
            for (int64_t i = 0; i < n; i++) { x[i] += alpha * p[i]; r[i] -= alpha * q[i]; }
            rel = std::sqrt(dot(r, r)) / bnorm;
            if (rel <= tol) { it++; break; }
            precondition(r.data(), z.data());
            const double rzNew = dot(r, z);
            const double beta = std::max(0.0, -alpha * dot(z, q) / rz);
            rz = rzNew;
            for (int64_t i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
        }
        apply<double>(0, x, q.data(), false);
        for (int64_t i = 0; i < n; i++) r[i] = L.fixed[i] ? 0 : f[i] - q[i];
        res.residual = std::sqrt(dot(r, r)) / bnorm;
        res.iterations = it;
        res.converged = std::isfinite(res.residual) && res.residual <= tol * 10;
        return res;
    }
};

// (voxel_fea.cpp:138-183)
static Model* build(const int dims[3], const float* density, double nu, const uint8_t* bc, int64_t coarsestMaxDof, const double* diagAdd) {
    if (dims[0] < 1 || dims[1] < 1 || dims[2] < 1) throw std::invalid_argument("The structural grid must have three positive dimensions.");
    const int64_t nE = int64_t(dims[0]) * dims[1] * dims[2];
    for (int64_t e = 0; e < nE; e++)
        if (!std::isfinite(density[e]) || density[e] < 0 || density[e] > 1) throw std::invalid_argument("Voxel density must be between zero and one.");
    auto* M = new Model;
    M->nu = nu;
    try {
        M->el = element(nu, true);
    } catch (...) {
        delete M;
        throw;
    }
    Level L0 = makeGrid(dims[0], dims[1], dims[2]);
    std::memcpy(L0.Kb, M->el.K, sizeof L0.Kb);
    L0.emap.assign(nE, -1);
    for (int64_t v = 0; v < nE; v++)
        if (density[v] > 0) {
            L0.emap[v] = int(L0.elems.size());
            L0.elems.push_back(int(v));
            L0.rho.push_back(density[v]);
        }
    L0.bc.assign(bc, bc + L0.nDof);
    if (diagAdd) L0.diagAdd.assign(diagAdd, diagAdd + L0.nDof);
    finish(L0);
    M->levels.push_back(std::move(L0));
    for (;;) {
        Level& L = M->levels.back();
        if (L.freeDof <= coarsestMaxDof || M->levels.size() >= 12) break;
        if (L.nx <= 1 && L.ny <= 1 && L.nz <= 1) break;
        Level C = coarsen(L);
        M->levels.push_back(std::move(C));
    }
    M->factorCoarsest();
    return M;
}

// ---- post-processing (voxel_fea.cpp:929-1119) ----

static double vonMises(const double* s) {
    return std::sqrt(0.5 * ((s[0] - s[1]) * (s[0] - s[1]) + (s[1] - s[2]) * (s[1] - s[2]) + (s[2] - s[0]) * (s[2] - s[0])) +
                     3 * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5]));
}

// eigenvalues of a symmetric 3x3 by the trigonometric method, descending (voxel_fea.cpp:947-966)
static void principal(double sx, double sy, double sz, double txy, double tyz, double tzx, double out[3]) {
    const double p1 = txy * txy + tyz * tyz + tzx * tzx;
    const double q = (sx + sy + sz) / 3;
    const double sc = std::fabs(sx) + std::fabs(sy) + std::fabs(sz) + std::sqrt(p1);
    if (p1 <= 1e-24 * sc * sc) {
        double v[3] = {sx, sy, sz};
        std::sort(v, v + 3, [](double a, double b) { return a > b; });
        out[0] = v[0]; out[1] = v[1]; out[2] = v[2];
        return;
    }
    const double p2 = (sx - q) * (sx - q) + (sy - q) * (sy - q) + (sz - q) * (sz - q) + 2 * p1;
    const double p = std::sqrt(p2 / 6);
    const double b11 = (sx - q) / p, b22 = (sy - q) / p, b33 = (sz - q) / p, b12 = txy / p, b23 = tyz / p, b13 = tzx / p;
    const double det = b11 * (b22 * b33 - b23 * b23) - b12 * (b12 * b33 - b23 * b13) + b13 * (b12 * b23 - b22 * b13);
    const double rr = std::min(1.0, std::max(-1.0, det / 2));
    const double phi = std::acos(rr) / 3;
    out[0] = q + 2 * p * std::cos(phi);
    out[2] = q + 2 * p * std::cos(phi + 2 * M_PI / 3);
    out[1] = 3 * q - out[0] - out[2];
}

// nodal von Mises / P1 / P3: rho-weighted mean of the surrounding voxels' corner stresses
// (voxel_fea.cpp:968-1037)
static void stresses(const Model& M, const double* u, double E, double h, bool principals, float* vm, float* p1, float* p3) {
    const Level& L = M.levels[0];
    for (int64_t n = 0; n < L.nNodes; n++) {
        vm[n] = 0;
        if (principals) { p1[n] = 0; p3[n] = 0; }
        if (!L.active[n]) continue;
        const int i = int(n % L.NX), j = int((n / L.NX) % L.NY), k = int(n / (int64_t(L.NX) * L.NY));
        double svm = 0, sp1 = 0, sp3 = 0, w = 0;
        for (int v = 0; v < 8; v++) {
            const int di = v & 1, dj = (v >> 1) & 1, dk = v >> 2;
            const int ei = i - 1 + di, ej = j - 1 + dj, ek = k - 1 + dk;
            if (ei < 0 || ej < 0 || ek < 0 || ei >= L.nx || ej >= L.ny || ek >= L.nz) continue;
            const int e = L.emap[ei + int64_t(L.nx) * (ej + int64_t(L.ny) * ek)];
            if (e < 0) continue;
            const int a = cornerOf(1 - di, 1 - dj, 1 - dk);
            double sig[6] = {0, 0, 0, 0, 0, 0};
            for (int b = 0; b < 8; b++) {
                const double* ub = u + 3 * L.node(ei + CORNER[b][0], ej + CORNER[b][1], ek + CORNER[b][2]);
                for (int r = 0; r < 6; r++)
                    for (int c = 0; c < 3; c++) sig[r] += M.el.cornerStress[a][r * 24 + 3 * b + c] * E / h * ub[c];
            }
            const double rho = L.rho[e];
            svm += rho * vonMises(sig);
            if (principals) {
                double pr[3];
                principal(sig[0], sig[1], sig[2], sig[3], sig[4], sig[5], pr);
                sp1 += rho * pr[0];
                sp3 += rho * pr[2];
            }
            w += rho;
        }
        if (w > 0) {
            vm[n] = float(svm / w);
            if (principals) { p1[n] = float(sp1 / w); p3[n] = float(sp3 / w); }
        }
    }
}

}  // namespace orc

// ---- C ABI for the Python test harness ----
extern "C" {

static void setErr(char* err, int len, const char* msg) {
    if (err && len > 0) { std::snprintf(err, size_t(len), "%s", msg); }
}

void* orc_create(const int32_t dims[3], const float* density, double nu, const uint8_t* bc, int64_t coarsest, const double* diag_add, char* err, int errlen) {
    try {
        const int d[3] = {dims[0], dims[1], dims[2]};
        return orc::build(d, density, nu, bc, coarsest, diag_add);
    } catch (const std::exception& e) {
        setErr(err, errlen, e.what());
        return nullptr;
    }
}
void orc_destroy(void* h) { delete static_cast<orc::Model*>(h); }
int orc_num_levels(void* h) { return int(static_cast<orc::Model*>(h)->levels.size()); }
// nx ny nz nNodes nDof freeDof nElems nOwn coarse_m
void orc_level_info(void* h, int l, int64_t* out) {
    auto* M = static_cast<orc::Model*>(h);
    const auto& L = M->levels[l];
    out[0] = L.nx; out[1] = L.ny; out[2] = L.nz; out[3] = L.nNodes; out[4] = L.nDof; out[5] = L.freeDof;
    out[6] = int64_t(L.elems.size()); out[7] = int64_t(L.own.size() / 576); out[8] = M->m;
}
void orc_level_fixed(void* h, int l, uint8_t* out) { auto& L = static_cast<orc::Model*>(h)->levels[l]; std::memcpy(out, L.fixed.data(), L.fixed.size()); }
void orc_level_active(void* h, int l, uint8_t* out) { auto& L = static_cast<orc::Model*>(h)->levels[l]; std::memcpy(out, L.active.data(), L.active.size()); }
void orc_level_kb(void* h, int l, double* out) { std::memcpy(out, static_cast<orc::Model*>(h)->levels[l].Kb, 576 * 8); }
void orc_level_elems(void* h, int l, int32_t* out) { auto& L = static_cast<orc::Model*>(h)->levels[l]; for (size_t e = 0; e < L.elems.size(); e++) out[e] = L.elems[e]; }
void orc_level_kidx(void* h, int l, int32_t* out) {
    auto& L = static_cast<orc::Model*>(h)->levels[l];
    for (size_t e = 0; e < L.elems.size(); e++) out[e] = L.kIdx.empty() ? -1 : L.kIdx[e];
}
void orc_level_rho(void* h, int l, double* out) { auto& L = static_cast<orc::Model*>(h)->levels[l]; std::memcpy(out, L.rho.data(), L.rho.size() * 8); }
void orc_level_own(void* h, int l, float* out) { auto& L = static_cast<orc::Model*>(h)->levels[l]; std::memcpy(out, L.own.data(), L.own.size() * 4); }
void orc_level_invdiag(void* h, int l, double* out) { auto& L = static_cast<orc::Model*>(h)->levels[l]; std::memcpy(out, L.invDiag.data(), L.invDiag.size() * 8); }
void orc_prepare(void* h) { static_cast<orc::Model*>(h)->prepare(); }
double orc_level_lmax(void* h, int l) { return static_cast<orc::Model*>(h)->levels[l].lmax; }
void orc_set_lmax(void* h, int l, double v) { auto& L = static_cast<orc::Model*>(h)->levels[l]; L.lmax = v; L.omega = 1.2 / (v * 1.05); }
void orc_apply(void* h, int l, const double* x, double* y, int raw) { static_cast<orc::Model*>(h)->apply<double>(l, x, y, raw != 0); }
void orc_apply32(void* h, int l, const float* x, float* y) { static_cast<orc::Model*>(h)->apply<float>(l, x, y, false); }
void orc_precondition(void* h, const double* r, double* z) {
    auto* M = static_cast<orc::Model*>(h);
    M->prepare();
    M->precondition(r, z);
}
// one V-cycle from level l with the given float32 right-hand side; z out (both nDof of level l)
void orc_vcycle32(void* h, int l, const float* r, float* z) {
    auto* M = static_cast<orc::Model*>(h);
    M->prepare();
    auto& L = M->levels[l];
    std::memcpy(L.r.data(), r, L.r.size() * 4);
    M->vcycle(l);
    std::memcpy(z, L.z.data(), L.z.size() * 4);
}
void orc_coarse_factor(void* h, double* out) { auto* M = static_cast<orc::Model*>(h); std::memcpy(out, M->chol.data(), M->chol.size() * 8); }
int orc_solve(void* h, const double* f, double tol, int max_iter, const double* x0, double* u, int32_t* iters, double* residual, int32_t* converged,
              char* err, int errlen) {
    try {
        auto r = static_cast<orc::Model*>(h)->solve(f, tol, max_iter, x0, u);
        *iters = r.iterations;
        *residual = r.residual;
        *converged = r.converged;
        return 0;
    } catch (const std::exception& e) {
        setErr(err, errlen, e.what());
        return 1;
    }
}
void orc_stresses(void* h, const double* u, double E, double hh, int principals, float* vm, float* p1, float* p3) {
    orc::stresses(*static_cast<orc::Model*>(h), u, E, hh, principals != 0, vm, p1, p3);
}
// support reactions: sum over held DOFs of active nodes of (K u - f) (voxel_fea.cpp:929-940)
void orc_reactions(void* h, const double* u, const double* f, double* R) {
    auto* M = static_cast<orc::Model*>(h);
    const auto& L = M->levels[0];
    std::vector<double> y(L.nDof);
    M->apply<double>(0, u, y.data(), true);
    R[0] = R[1] = R[2] = 0;
    for (int64_t n = 0; n < L.nNodes; n++)
        for (int d = 0; d < 3; d++)
            if (L.bc[3 * n + d] && L.active[n]) R[d] += y[3 * n + d] - (f ? f[3 * n + d] : 0.0);
}
int orc_element(double nu, int modes, double* K, double* cornerStress, double* gaussB, char* err, int errlen) {
    try {
        const auto el = orc::element(nu, modes != 0);
        std::memcpy(K, el.K, sizeof el.K);
        if (cornerStress) std::memcpy(cornerStress, el.cornerStress, sizeof el.cornerStress);
        if (gaussB) std::memcpy(gaussB, el.gaussB, sizeof el.gaussB);
        return 0;
    } catch (const std::exception& e) {
        setErr(err, errlen, e.what());
        return 1;
    }
}
// voxels face-connected to a voxel touching a held node survive (voxel_fea.cpp:1086-1119)
int orc_prune(const int32_t dims[3], const float* density, const uint8_t* heldNode, float* out) {
    const int nx = dims[0], ny = dims[1], nz = dims[2];
    const int64_t NX = nx + 1, NY = ny + 1, nE = int64_t(nx) * ny * nz;
    std::vector<uint8_t> seen(nE, 0);
    std::vector<int64_t> queue;
    for (int64_t e = 0; e < nE; e++) {
        if (!(density[e] > 0)) continue;
        const int i = int(e % nx), j = int((e / nx) % ny), k = int(e / (int64_t(nx) * ny));
        for (int a = 0; a < 8 && !seen[e]; a++)
            if (heldNode[(i + orc::CORNER[a][0]) + NX * ((j + orc::CORNER[a][1]) + NY * (k + orc::CORNER[a][2]))]) { seen[e] = 1; queue.push_back(e); }
    }
    for (size_t q = 0; q < queue.size(); q++) {
        const int64_t e = queue[q];
        const int i = int(e % nx), j = int((e / nx) % ny), k = int(e / (int64_t(nx) * ny));
        const int64_t nb[6] = {i > 0 ? e - 1 : -1, i < nx - 1 ? e + 1 : -1, j > 0 ? e - nx : -1, j < ny - 1 ? e + nx : -1,
                               k > 0 ? e - int64_t(nx) * ny : -1, k < nz - 1 ? e + int64_t(nx) * ny : -1};
        for (int64_t m : nb)
            if (m >= 0 && !seen[m] && density[m] > 0) { seen[m] = 1; queue.push_back(m); }
    }
    int removed = 0;
    for (int64_t e = 0; e < nE; e++) {
        out[e] = (density[e] > 0 && seen[e]) ? density[e] : 0.f;
        if (density[e] > 0 && !seen[e]) removed++;
    }
    return removed;
}

}  // extern "C"
