// The unit-cube hex8 element shared by every voxel (E = 1, side 1).
#pragma once

namespace psfea {

// corner a of a voxel at unit offset CORNER_XYZ[a] (bottom face counter-clockwise, then top face;
// the node order of native/src/fea/hex8.hpp:14)
constexpr int CORNER_XYZ[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};

// corner index of the unit offset (x, y, z), each 0 or 1
constexpr int cornerIndex(int x, int y, int z) { return (y ? (x ? 2 : 3) : (x ? 1 : 0)) + 4 * z; }

struct HexElement {
    double K[576];                 // condensed 24x24 stiffness, row-major, DOF 3a + d
    double cornerStress[8][144];   // D * Bbar at each corner (6 x 24)
};

// Wilson incompatible-mode hex8 (9 bubble modes condensed statically) on a 2x2x2 Gauss rule,
// symmetrised; or the plain trilinear element when incompatibleModes is false.
// Follows native/src/fea/hex8.cpp:104-155. Throws Error(PS_EINVAL) for nu outside (-1, 0.5).
HexElement hexElement(double nu, bool incompatibleModes = true);

}  // namespace psfea
