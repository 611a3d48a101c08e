// Host-side multigrid hierarchy build. Rules (not code) of native/src/fea/voxel_fea.cpp:
//   level 0 from the voxel densities ............................ :138-171
//   fixed mask = !active | bc | !(diag > 0), free DOFs ........... :208-234
//   uniform (27-point stencil) nodes ............................. :249-261
//   2:1 coarsening, (n + 1) >> 1 per axis ......................... :268-269
//   coarse uniform element Kb = sum over child positions of
//   P_c^T Kb P_c; a coarse element whose 8 children are the same
//   s * Kb is s * Kb_coarse, every other one gets its own exact
//   Galerkin matrix, numbered in increasing coarse-voxel order ... :309-354
//   coarse held DOF = OR of the fine held DOFs it interpolates to . :355-378
//   diagAdd restricted as P^T d ................................... :379-383
//   stop when free DOFs <= coarsestMaxDof, 12 levels, or 1x1x1 .... :174-180
//   coarsest dense matrix, Cholesky with tiny pivots replaced by
//   the largest diagonal, none when m == 0 or m > 3000 ........... :612-661
// Everything runs over all host cores; the result does not depend on the thread count. An optional
// engine (galerkin.cu) forms the own matrices of graded levels on the device, bitwise the same.
#include "hierarchy.hpp"

#include <cmath>
#include <cstring>
#include <unordered_map>

#include "host_util.hpp"

namespace psfea {

namespace {

inline uint32_t floatBits(float s) {
    uint32_t w;
    std::memcpy(&w, &s, 4);
    return w;
}
inline float bitsFloat(uint32_t w) {
    float s;
    std::memcpy(&s, &w, 4);
    return s;
}

HostLevel makeGrid(int nx, int ny, int nz) {
    HostLevel L;
    L.nx = nx; L.ny = ny; L.nz = nz;
    L.NX = nx + 1; L.NY = ny + 1; L.NZ = nz + 1;
    L.nVox = int64_t(nx) * ny * nz;
    L.nNodes = int64_t(L.NX) * L.NY * L.NZ;
    L.nDof = 3 * L.nNodes;
    return L;
}

// Kb and its 27-point stencil. Node n is corner a = (1-di, 1-dj, 1-dk) of the voxel at offset
// (di, dj, dk) - 1; that voxel's corner b is the neighbour at offset (di + bx - 1, ...).
void setBase(HostLevel& L, const double* K) {
    std::memcpy(L.Kb, K, sizeof L.Kb);
    std::memset(L.S, 0, sizeof L.S);
    for (int v = 0; v < 8; v++) {
        const int di = v & 1, dj = (v >> 1) & 1, dk = v >> 2;
        const int a = cornerIndex(1 - di, 1 - dj, 1 - dk);
        for (int b = 0; b < 8; b++) {
            const int ox = di + CORNER_XYZ[b][0] - 1, oy = dj + CORNER_XYZ[b][1] - 1, oz = dk + CORNER_XYZ[b][2] - 1;
            const int m = (ox + 1) + 3 * (oy + 1) + 9 * (oz + 1);
            for (int d = 0; d < 3; d++)
                for (int c = 0; c < 3; c++) L.S[m][3 * d + c] += K[(3 * a + d) * 24 + 3 * b + c];
        }
    }
}

// matrix entry (r, c) of the element held in voxel word w, as a double
inline double entry(const HostLevel& L, uint32_t w, int r, int c) {
    if (w & OWN_BIT) return double(L.own[int64_t(w & ~OWN_BIT) * 576 + r * 24 + c]);
    return double(bitsFloat(w)) * L.Kb[r * 24 + c];
}

// diagonal, masks, inverse diagonal, uniform flags and the boundary node list
void finishLevel(HostLevel& L) {
    // both written in full below (one pass per z plane), so allocated without a serial zero fill
    L.nmask.resize(size_t(L.nNodes));
    L.invDiag.resize(size_t(L.nDof));
    std::vector<int64_t> freeCount(size_t(L.NZ), 0);
    parallelFor(L.NZ, [&](int64_t k0, int64_t k1) {
        for (int64_t k = k0; k < k1; k++) {
            int64_t nfree = 0;
            for (int j = 0; j < L.NY; j++)
                for (int i = 0; i < L.NX; i++) {
                    const int64_t n = L.node(i, j, int(k));
                    double diag[3] = {0, 0, 0};
                    bool active = false;
                    uint32_t w0 = 0;
                    bool uniform = true;
                    for (int v = 0; v < 8; v++) {
                        const int di = v & 1, dj = (v >> 1) & 1, dk = v >> 2;
                        const int ei = i - 1 + di, ej = j - 1 + dj, ek = int(k) - 1 + dk;
                        uint32_t w = 0;
                        if (ei >= 0 && ej >= 0 && ek >= 0 && ei < L.nx && ej < L.ny && ek < L.nz) w = L.word[L.voxel(ei, ej, ek)];
                        if (v == 0) w0 = w;
                        uniform = uniform && w == w0;
                        if (!w) continue;
                        active = true;
                        const int a = cornerIndex(1 - di, 1 - dj, 1 - dk);
                        for (int d = 0; d < 3; d++) diag[d] += entry(L, w, 3 * a + d, 3 * a + d);
                    }
                    uint8_t m = 0;
                    if (active) {
                        m |= NM_ACTIVE;
                        if (uniform && w0 && !(w0 & OWN_BIT)) m |= NM_UNIFORM;
                    }
                    for (int d = 0; d < 3; d++) {
                        double dg = diag[d];
                        if (!L.diagAdd.empty()) dg += L.diagAdd[3 * n + d];
                        if (!active || L.bc[3 * n + d] || !(dg > 0)) {
                            m |= uint8_t(1u << d);
                            L.invDiag[3 * n + d] = 0.0;
                        } else {
                            L.invDiag[3 * n + d] = 1 / dg;
                            nfree++;
                        }
                    }
                    L.nmask[n] = m;
                }
            freeCount[size_t(k)] = nfree;
        }
    }, 1);
    L.freeDof = 0;
    for (auto c : freeCount) L.freeDof += c;
    L.boundary.clear();
    for (int64_t n = 0; n < L.nNodes; n++)
        if ((L.nmask[n] & NM_ACTIVE) && !(L.nmask[n] & NM_UNIFORM)) L.boundary.push_back(int32_t(n));
}

// interpolation weight of coarse corner b at corner a of the fine child in position c
double childWeight(int c, int a, int b) {
    double w = 1;
    for (int d = 0; d < 3; d++) {
        const double s = (((c >> d) & 1) + CORNER_XYZ[a][d]) * 0.5;
        w *= CORNER_XYZ[b][d] ? s : 1 - s;
    }
    return w;
}

struct ChildWeights {
    double W[8][8][8];  // [c][a][b]
    ChildWeights() {
        for (int c = 0; c < 8; c++)
            for (int a = 0; a < 8; a++)
                for (int b = 0; b < 8; b++) W[c][a][b] = childWeight(c, a, b);
    }
};
const ChildWeights& childWeights() {
    static const ChildWeights cw;
    return cw;
}

// out += s * P_c^T K P_c with P_c[3a + d][3b + d] = W[c][a][b]
void galerkinAdd(double* out, const double* K, int c, double s) {
    const auto& W = childWeights().W[c];
    double T[576];  // K P_c
    for (int r = 0; r < 24; r++)
        for (int b = 0; b < 8; b++) {
            double t0 = 0, t1 = 0, t2 = 0;
            for (int a = 0; a < 8; a++) {
                const double w = W[a][b];
                if (w == 0) continue;
                const double* kr = K + r * 24 + 3 * a;
                t0 += kr[0] * w;
                t1 += kr[1] * w;
                t2 += kr[2] * w;
            }
            T[r * 24 + 3 * b] = t0;
            T[r * 24 + 3 * b + 1] = t1;
            T[r * 24 + 3 * b + 2] = t2;
        }
    for (int b = 0; b < 8; b++)
        for (int a = 0; a < 8; a++) {
            const double w = W[a][b] * s;
            if (w == 0) continue;
            for (int d = 0; d < 3; d++) {
                double* o = out + (3 * b + d) * 24;
                const double* t = T + (3 * a + d) * 24;
                for (int q = 0; q < 24; q++) o[q] += w * t[q];
            }
        }
}

HostLevel coarsen(const HostLevel& F, GalerkinEngine* engine) {
    HostLevel C = makeGrid((F.nx + 1) >> 1, (F.ny + 1) >> 1, (F.nz + 1) >> 1);
    double M[8][576];
    double Kc[576] = {};
    for (int c = 0; c < 8; c++) {
        std::memset(M[c], 0, sizeof M[c]);
        galerkinAdd(M[c], F.Kb, c, 1.0);
        for (int u = 0; u < 576; u++) Kc[u] += M[c][u];
    }
    setBase(C, Kc);
    // classify every coarse voxel: empty / uniform (same word as its 8 children) / own matrix
    C.word.assign(C.nVox, 0);
    std::vector<uint8_t> isOwn(C.nVox, 0);
    auto childWord = [&](int I, int J, int K, int c) -> uint32_t {
        const int i = 2 * I + (c & 1), j = 2 * J + ((c >> 1) & 1), k = 2 * K + (c >> 2);
        if (i >= F.nx || j >= F.ny || k >= F.nz) return 0;
        return F.word[F.voxel(i, j, k)];
    };
    parallelFor(C.nz, [&](int64_t k0, int64_t k1) {
        for (int64_t K = k0; K < k1; K++)
            for (int J = 0; J < C.ny; J++)
                for (int I = 0; I < C.nx; I++) {
                    uint32_t w0 = childWord(I, J, int(K), 0);
                    bool any = false, uniform = w0 != 0 && !(w0 & OWN_BIT);
                    for (int c = 0; c < 8; c++) {
                        const uint32_t w = childWord(I, J, int(K), c);
                        any = any || w != 0;
                        uniform = uniform && w == w0;
                    }
                    const int64_t v = C.voxel(I, J, int(K));
                    if (uniform) C.word[v] = w0;
                    else if (any) isOwn[v] = 1;
                }
    }, 1);
    int64_t nOwn = 0;
    std::vector<int64_t> ownVox;  // the voxel of each own matrix, in increasing voxel order
    for (int64_t v = 0; v < C.nVox; v++) {
        if (isOwn[v]) {
            C.word[v] = OWN_BIT | uint32_t(nOwn++);
            ownVox.push_back(v);
        }
        if (isOwn[v] || C.word[v]) C.nElems++;
    }
    C.nOwn = nOwn;
    C.own.resize(size_t(nOwn) * 576);  // every matrix is written below (its class's first voxel computes it)
    // the Galerkin matrix of own coarse voxel v, stored 32-bit at dst
    auto computeOwn = [&](int64_t v, double* out, double* Kf, float* dst) {
        const int I = int(v % C.nx), J = int((v / C.nx) % C.ny), K = int(v / (int64_t(C.nx) * C.ny));
        std::fill(out, out + 576, 0.0);
        for (int c = 0; c < 8; c++) {
            const uint32_t w = childWord(I, J, K, c);
            if (!w) continue;
            if (w & OWN_BIT) {
                const float* src = F.own.data() + int64_t(w & ~OWN_BIT) * 576;
                for (int u = 0; u < 576; u++) Kf[u] = double(src[u]);
                galerkinAdd(out, Kf, c, 1.0);
            } else {
                const double s = double(bitsFloat(w));
                for (int u = 0; u < 576; u++) out[u] += s * M[c][u];
            }
        }
        for (int u = 0; u < 576; u++) dst[u] = float(out[u]);
    };
    // Own coarse voxels whose 8 children match (empty, the same uniform word, or own matrices of
    // one class) have bitwise the same matrix: each class is computed once, at its first voxel, by
    // the code above, and copied to the others. Lattices and solid/void parts have a few hundred
    // classes over millions of voxels; on graded grids (nearly all distinct) the search stops
    // after a sample and every voxel is its own class.
    struct ChildKey {
        uint64_t d[8];
        bool operator==(const ChildKey& o) const { return std::memcmp(d, o.d, sizeof d) == 0; }
    };
    struct ChildKeyHash {
        size_t operator()(const ChildKey& k) const {
            uint64_t h = 0x9e3779b97f4a7c15ull;
            for (uint64_t v : k.d) {
                h ^= v + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
                h *= 0xff51afd7ed558ccdull;
            }
            return size_t(h ^ (h >> 32));
        }
    };
    std::vector<ChildKey> keys(static_cast<size_t>(nOwn));
    parallelFor(nOwn, [&](int64_t o0, int64_t o1) {
        for (int64_t o = o0; o < o1; o++) {
            const int64_t v = ownVox[size_t(o)];
            const int I = int(v % C.nx), J = int((v / C.nx) % C.ny), K = int(v / (int64_t(C.nx) * C.ny));
            for (int c = 0; c < 8; c++) {
                const uint32_t w = childWord(I, J, K, c);
                keys[size_t(o)].d[c] = !w ? 0 : (w & OWN_BIT) ? ((uint64_t(2) << 32) | uint32_t(F.ownClass[w & ~OWN_BIT])) : ((uint64_t(1) << 32) | w);
            }
        }
    }, 4096);
    C.ownClass.assign(size_t(nOwn), 0);
    std::vector<int64_t> rep;  // the first own index of each class
    {
        std::unordered_map<ChildKey, int32_t, ChildKeyHash> classOf;
        const int64_t sample = std::min<int64_t>(nOwn, int64_t(1) << 16);
        bool shared = true;
        for (int64_t o = 0; o < nOwn; o++) {
            const auto it = classOf.try_emplace(keys[size_t(o)], int32_t(rep.size()));
            if (it.second) rep.push_back(o);
            C.ownClass[size_t(o)] = it.first->second;
            if (o + 1 == sample && int64_t(rep.size()) * 2 > sample) {
                shared = false;
                break;
            }
        }
        if (!shared) {
            rep.resize(size_t(nOwn));
            for (int64_t o = 0; o < nOwn; o++) {
                rep[size_t(o)] = o;
                C.ownClass[size_t(o)] = int32_t(o);
            }
        }
    }
    if (engine && nOwn > 0 && int64_t(rep.size()) >= engine->minClasses()) {
        // every own matrix (class members included: they come out bitwise equal to their class's)
        engine->computeOwn(F, C, ownVox, M, C.own.data());
    } else {
        parallelFor(int64_t(rep.size()), [&](int64_t c0, int64_t c1) {
            std::vector<double> out(576), Kf(576);
            for (int64_t c = c0; c < c1; c++) {
                const int64_t o = rep[size_t(c)];
                computeOwn(ownVox[size_t(o)], out.data(), Kf.data(), C.own.data() + o * 576);
            }
        }, 256);
    }
    parallelFor(nOwn, [&](int64_t o0, int64_t o1) {
        for (int64_t o = o0; o < o1; o++) {
            const int64_t r = rep[size_t(C.ownClass[size_t(o)])];
            if (r != o) std::memcpy(C.own.data() + o * 576, C.own.data() + r * 576, 576 * sizeof(float));
        }
    }, 4096);
    // held coarse DOFs: fine node i interpolates to coarse i/2 and, when odd, (i+1)/2
    C.bc.assign(C.nDof, 0);
    parallelFor(C.NZ, [&](int64_t K0, int64_t K1) {
        for (int64_t K = K0; K < K1; K++)
            for (int J = 0; J < C.NY; J++)
                for (int I = 0; I < C.NX; I++) {
                    uint8_t b[3] = {0, 0, 0};
                    for (int k = int(2 * K - 1); k <= int(2 * K + 1); k++) {
                        if (k < 0 || k >= F.NZ) continue;
                        for (int j = 2 * J - 1; j <= 2 * J + 1; j++) {
                            if (j < 0 || j >= F.NY) continue;
                            for (int i = 2 * I - 1; i <= 2 * I + 1; i++) {
                                if (i < 0 || i >= F.NX) continue;
                                const uint8_t* fb = F.bc.data() + 3 * F.node(i, j, k);
                                b[0] |= fb[0];
                                b[1] |= fb[1];
                                b[2] |= fb[2];
                            }
                        }
                    }
                    uint8_t* cb = C.bc.data() + 3 * C.node(I, J, int(K));
                    cb[0] = b[0]; cb[1] = b[1]; cb[2] = b[2];
                }
    }, 1);
    if (!F.diagAdd.empty()) {
        C.diagAdd.assign(C.nDof, 0.0);
        parallelFor(C.nNodes, [&](int64_t lo, int64_t hi) {
            for (int64_t cn = lo; cn < hi; cn++) {
                const int I = int(cn % C.NX), J = int((cn / C.NX) % C.NY), K = int(cn / (int64_t(C.NX) * C.NY));
                double s[3] = {0, 0, 0};
                for (int dk = -1; dk <= 1; dk++)
                    for (int dj = -1; dj <= 1; dj++)
                        for (int di = -1; di <= 1; di++) {
                            const int i = 2 * I + di, j = 2 * J + dj, k = 2 * K + dk;
                            if (i < 0 || j < 0 || k < 0 || i >= F.NX || j >= F.NY || k >= F.NZ) continue;
                            const double w = (di ? 0.5 : 1.0) * (dj ? 0.5 : 1.0) * (dk ? 0.5 : 1.0);
                            for (int d = 0; d < 3; d++) s[d] += w * F.diagAdd[3 * F.node(i, j, k) + d];
                        }
                for (int d = 0; d < 3; d++) C.diagAdd[3 * cn + d] = s[d];
            }
        });
    }
    finishLevel(C);
    return C;
}

void buildCoarsest(Hierarchy& H) {
    const HostLevel& L = H.levels.back();
    std::vector<int64_t> map(L.nDof, -1);
    int64_t m = 0;
    for (int64_t i = 0; i < L.nDof; i++)
        if (!L.fixedDof(i)) map[i] = m++;
    H.coarseM = m;
    H.coarseDof.clear();
    H.coarseInv.clear();
    H.coarseChol.clear();
    if (m == 0 || m > 3000) return;
    H.coarseDof.resize(size_t(m));
    for (int64_t i = 0; i < L.nDof; i++)
        if (map[i] >= 0) H.coarseDof[size_t(map[i])] = int32_t(i);
    std::vector<double>& A = H.coarseChol;
    A.assign(size_t(m * m), 0.0);
    for (int k = 0; k < L.nz; k++)
        for (int j = 0; j < L.ny; j++)
            for (int i = 0; i < L.nx; i++) {
                const uint32_t w = L.word[L.voxel(i, j, k)];
                if (!w) continue;
                int64_t dofs[24];
                for (int a = 0; a < 8; a++)
                    for (int d = 0; d < 3; d++)
                        dofs[3 * a + d] = map[3 * L.node(i + CORNER_XYZ[a][0], j + CORNER_XYZ[a][1], k + CORNER_XYZ[a][2]) + d];
                for (int r = 0; r < 24; r++) {
                    if (dofs[r] < 0) continue;
                    for (int c = 0; c < 24; c++)
                        if (dofs[c] >= 0) A[size_t(dofs[r] * m + dofs[c])] += entry(L, w, r, c);
                }
            }
    if (!L.diagAdd.empty())
        for (int64_t i = 0; i < L.nDof; i++)
            if (map[i] >= 0) A[size_t(map[i] * m + map[i])] += L.diagAdd[i];
    double maxDiag = 0;
    for (int64_t i = 0; i < m; i++) maxDiag = std::max(maxDiag, A[size_t(i * m + i)]);
    // right-looking Cholesky, the trailing rows updated in parallel
    for (int64_t j = 0; j < m; j++) {
        double s = A[size_t(j * m + j)];
        if (!(s > 1e-10 * maxDiag)) s = maxDiag;  // a near-mechanism at the coarsest level
        const double ljj = std::sqrt(s), inv = 1 / ljj;
        A[size_t(j * m + j)] = ljj;
        for (int64_t i = j + 1; i < m; i++) A[size_t(i * m + j)] *= inv;
        parallelFor(m - j - 1, [&](int64_t lo, int64_t hi) {
            for (int64_t ii = lo; ii < hi; ii++) {
                const int64_t i = j + 1 + ii;
                const double lij = A[size_t(i * m + j)];
                if (lij == 0) continue;
                double* row = A.data() + i * m;
                for (int64_t k = j + 1; k <= i; k++) row[k] -= lij * A[size_t(k * m + j)];
            }
        }, 64);
    }
    for (int64_t i = 0; i < m; i++)
        for (int64_t k = i + 1; k < m; k++) A[size_t(i * m + k)] = 0;
    // dense inverse, one column per task: L y = e_c, then L^T x = y
    H.coarseInv.assign(size_t(m * m), 0.0);
    parallelFor(m, [&](int64_t c0, int64_t c1) {
        std::vector<double> y(static_cast<size_t>(m));
        for (int64_t c = c0; c < c1; c++) {
            std::fill(y.begin(), y.end(), 0.0);
            y[size_t(c)] = 1;
            for (int64_t i = c; i < m; i++) {
                double s = y[size_t(i)];
                const double* row = A.data() + i * m;
                for (int64_t k = c; k < i; k++) s -= row[k] * y[size_t(k)];
                y[size_t(i)] = s / row[i];
            }
            for (int64_t i = m - 1; i >= 0; i--) {
                double s = y[size_t(i)];
                for (int64_t k = i + 1; k < m; k++) s -= A[size_t(k * m + i)] * y[size_t(k)];
                y[size_t(i)] = s / A[size_t(i * m + i)];
            }
            for (int64_t i = 0; i < m; i++) H.coarseInv[size_t(i * m + c)] = y[size_t(i)];
        }
    }, 4);
}

}  // namespace

double tridiagonalMax(const std::vector<double>& a, const std::vector<double>& b) {
    const int k = int(a.size());
    double lo = INFINITY, hi = -INFINITY;
    for (int i = 0; i < k; i++) {
        const double r = (i > 0 ? std::fabs(b[size_t(i - 1)]) : 0) + (i + 1 < k ? std::fabs(b[size_t(i)]) : 0);
        lo = std::min(lo, a[size_t(i)] - r);
        hi = std::max(hi, a[size_t(i)] + r);
    }
    // Sturm count: eigenvalues above x = positive pivots of T - x I
    auto above = [&](double x) {
        int count = 0;
        double q = 1;
        for (int i = 0; i < k; i++) {
            q = a[size_t(i)] - x - (i > 0 ? b[size_t(i - 1)] * b[size_t(i - 1)] / q : 0);
            if (q == 0) q = 1e-300;
            if (q > 0) count++;
        }
        return count;
    };
    for (int it = 0; it < 100 && hi - lo > 1e-12 * std::fabs(hi); it++) {
        const double mid = 0.5 * (lo + hi);
        if (above(mid) > 0) lo = mid;
        else hi = mid;
    }
    return hi;
}

void chebyshevCoefficients(double lmax, double& first, double& c1, double& c2) {
    const double b = 1.15 * lmax, a = 0.1 * lmax;
    const double theta = (b + a) / 2, delta = (b - a) / 2, sigma = theta / delta;
    const double rho0 = 1 / sigma, rho1 = 1 / (2 * sigma - rho0);
    first = 1 / theta;
    c1 = rho1 * rho0;
    c2 = 2 * rho1 / delta;
}

Hierarchy buildHierarchy(const int32_t dims[3], const float* density, double nu, const uint8_t* bc, int64_t coarsestMaxDof,
                         const double* diagAdd, GalerkinEngine* engine) {
    if (dims[0] < 1 || dims[1] < 1 || dims[2] < 1) throw Error(PS_EINVAL, "The structural grid must have three positive dimensions.");
    if (int64_t(dims[0] + 1) * (dims[1] + 1) * (dims[2] + 1) >= (int64_t(1) << 31))
        throw Error(PS_EINVAL, "The structural grid has more than 2^31 nodes.");
    if (!density || !bc) throw Error(PS_EINVAL, "Structural grid, density and fixture sizes do not match.");
    Hierarchy H;
    H.nu = nu;
    H.el = hexElement(nu);
    HostLevel L0 = makeGrid(dims[0], dims[1], dims[2]);
    {
        bool bad = false;
        L0.word.assign(L0.nVox, 0);
        for (int64_t v = 0; v < L0.nVox; v++) {
            const float r = density[v];
            if (!std::isfinite(r) || r < 0 || r > 1) bad = true;
            else if (r > 0) {
                L0.word[v] = floatBits(r);
                L0.nElems++;
            }
        }
        if (bad) throw Error(PS_EINVAL, "Voxel density must be between zero and one.");
    }
    setBase(L0, H.el.K);
    L0.bc.assign(bc, bc + L0.nDof);
    if (diagAdd) L0.diagAdd.assign(diagAdd, diagAdd + L0.nDof);
    finishLevel(L0);
    H.levels.push_back(std::move(L0));
    for (;;) {
        const HostLevel& L = H.levels.back();
        if (L.freeDof <= coarsestMaxDof || H.levels.size() >= 12) break;
        if (L.nx <= 1 && L.ny <= 1 && L.nz <= 1) break;
        HostLevel C = coarsen(L, engine);
        H.levels.push_back(std::move(C));
    }
    buildCoarsest(H);
    return H;
}

}  // namespace psfea
