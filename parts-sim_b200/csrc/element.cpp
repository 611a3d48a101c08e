// Unit-cube hex8 element. The formulation follows native/src/fea/hex8.cpp:8-155: isotropic D for
// E = 1 (hex8.cpp:8-18), strain-displacement rows from trilinear shape gradients (hex8.cpp:32-43),
// Wilson bubble modes 1 - xi^2 etc. (hex8.cpp:46-51), static condensation
// K = Kuu - Kua Kaa^-1 Kau (hex8.cpp:121-135), and corner stresses D (B + G A) (hex8.cpp:137-154).
// Here Kaa (symmetric positive definite) is factorised by Cholesky.
#include "element.hpp"

#include <cmath>
#include <cstring>

#include "host_util.hpp"

namespace psfea {

namespace {


// strain rows 0..5 (xx, yy, zz, xy, yz, zx with engineering shear) of a displacement triple whose
// shape function has gradient (gx, gy, gz), written into columns c..c+2 of M (ncol columns)
void strainOf(double* M, int ncol, int c, double gx, double gy, double gz) {
    M[0 * ncol + c + 0] = gx;
    M[1 * ncol + c + 1] = gy;
    M[2 * ncol + c + 2] = gz;
    M[3 * ncol + c + 0] = gy;
    M[3 * ncol + c + 1] = gx;
    M[4 * ncol + c + 1] = gz;
    M[4 * ncol + c + 2] = gy;
    M[5 * ncol + c + 0] = gz;
    M[5 * ncol + c + 2] = gx;
}

// B at natural coordinates p in [-1, 1]^3; the unit cube maps with dx/dxi = 1/2
void shapeStrain(const double p[3], double B[144]) {
    std::memset(B, 0, 144 * sizeof(double));
    for (int a = 0; a < 8; a++) {
        double s[3], f[3];
        for (int d = 0; d < 3; d++) {
            s[d] = 2.0 * CORNER_XYZ[a][d] - 1;
            f[d] = 1 + s[d] * p[d];
        }
        // N_a = f0 f1 f2 / 8, dN/dx_d = 2 * dN/dxi_d
        strainOf(B, 24, 3 * a, s[0] * f[1] * f[2] / 4, s[1] * f[0] * f[2] / 4, s[2] * f[0] * f[1] / 4);
    }
}

// strains of the 9 bubble amplitudes (6 x 9): mode m of component d has gradient -4 p_m e_m
void bubbleStrain(const double p[3], double G[54]) {
    std::memset(G, 0, 54 * sizeof(double));
    for (int m = 0; m < 3; m++) {
        double g[3] = {0, 0, 0};
        g[m] = -4 * p[m];
        strainOf(G, 9, 3 * m, g[0], g[1], g[2]);
    }
}

}  // namespace

HexElement hexElement(double nu, bool modes) {
    if (!std::isfinite(nu) || nu <= -1 || nu >= 0.5) throw Error(PS_EINVAL, "Poisson's ratio must be greater than -1 and less than 0.5.");
    double D[6][6] = {};
    const double lam = nu / ((1 + nu) * (1 - 2 * nu)), mu = 1 / (2 * (1 + nu));
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) D[i][j] = lam + (i == j ? 2 * mu : 0);
    for (int i = 3; i < 6; i++) D[i][i] = mu;

    const double g = 1 / std::sqrt(3.0), weight = 1.0 / 8;  // Jacobian determinant of the unit cube
    double kuu[576] = {}, kua[216] = {}, kaa[81] = {};
    for (int q = 0; q < 8; q++) {
        const double p[3] = {CORNER_XYZ[q][0] ? g : -g, CORNER_XYZ[q][1] ? g : -g, CORNER_XYZ[q][2] ? g : -g};
        double B[144], G[54], DB[144], DG[54];
        shapeStrain(p, B);
        bubbleStrain(p, G);
        for (int r = 0; r < 6; r++) {
            for (int c = 0; c < 24; c++) {
                double s = 0;
                for (int k = 0; k < 6; k++) s += D[r][k] * B[k * 24 + c];
                DB[r * 24 + c] = s;
            }
            for (int c = 0; c < 9; c++) {
                double s = 0;
                for (int k = 0; k < 6; k++) s += D[r][k] * G[k * 9 + c];
                DG[r * 9 + c] = s;
            }
        }
        for (int i = 0; i < 24; i++) {
            for (int j = 0; j < 24; j++) {
                double s = 0;
                for (int k = 0; k < 6; k++) s += B[k * 24 + i] * DB[k * 24 + j];
                kuu[i * 24 + j] += weight * s;
            }
            for (int j = 0; j < 9; j++) {
                double s = 0;
                for (int k = 0; k < 6; k++) s += B[k * 24 + i] * DG[k * 9 + j];
                kua[i * 9 + j] += weight * s;
            }
        }
        for (int i = 0; i < 9; i++)
            for (int j = 0; j < 9; j++) {
                double s = 0;
                for (int k = 0; k < 6; k++) s += G[k * 9 + i] * DG[k * 9 + j];
                kaa[i * 9 + j] += weight * s;
            }
    }
    // amplitudes alpha = A u with A = -Kaa^-1 Kau (9 x 24), by Cholesky of Kaa
    double A[216] = {};
    if (modes) {
        double L[81] = {};
        for (int j = 0; j < 9; j++) {
            double s = kaa[j * 9 + j];
            for (int k = 0; k < j; k++) s -= L[j * 9 + k] * L[j * 9 + k];
            L[j * 9 + j] = std::sqrt(s);
            for (int i = j + 1; i < 9; i++) {
                double t = kaa[i * 9 + j];
                for (int k = 0; k < j; k++) t -= L[i * 9 + k] * L[j * 9 + k];
                L[i * 9 + j] = t / L[j * 9 + j];
            }
        }
        for (int c = 0; c < 24; c++) {
            double y[9];
            for (int i = 0; i < 9; i++) {
                double s = -kua[c * 9 + i];
                for (int k = 0; k < i; k++) s -= L[i * 9 + k] * y[k];
                y[i] = s / L[i * 9 + i];
            }
            for (int i = 8; i >= 0; i--) {
                double s = y[i];
                for (int k = i + 1; k < 9; k++) s -= L[k * 9 + i] * y[k];
                y[i] = s / L[i * 9 + i];
            }
            for (int i = 0; i < 9; i++) A[i * 24 + c] = y[i];
        }
        for (int i = 0; i < 24; i++)
            for (int j = 0; j < 24; j++) {
                double s = 0;
                for (int q = 0; q < 9; q++) s += kua[i * 9 + q] * A[q * 24 + j];
                kuu[i * 24 + j] += s;
            }
        for (int i = 0; i < 24; i++)
            for (int j = i + 1; j < 24; j++) kuu[i * 24 + j] = kuu[j * 24 + i] = 0.5 * (kuu[i * 24 + j] + kuu[j * 24 + i]);
    }
    HexElement el;
    std::memcpy(el.K, kuu, sizeof kuu);
    for (int a = 0; a < 8; a++) {
        const double p[3] = {2.0 * CORNER_XYZ[a][0] - 1, 2.0 * CORNER_XYZ[a][1] - 1, 2.0 * CORNER_XYZ[a][2] - 1};
        double B[144], G[54];
        shapeStrain(p, B);
        if (modes) {
            bubbleStrain(p, G);
            for (int r = 0; r < 6; r++)
                for (int c = 0; c < 24; c++) {
                    double s = 0;
                    for (int q = 0; q < 9; q++) s += G[r * 9 + q] * A[q * 24 + c];
                    B[r * 24 + c] += s;
                }
        }
        for (int r = 0; r < 6; r++)
            for (int c = 0; c < 24; c++) {
                double s = 0;
                for (int k = 0; k < 6; k++) s += D[r][k] * B[k * 24 + c];
                el.cornerStress[a][r * 24 + c] = s;
            }
    }
    return el;
}

}  // namespace psfea
