// Host-side helpers shared between the library's translation units (not part
// of the C ABI).
#pragma once

#include <cstdint>
#include <vector>

namespace gbfk_host {

// One cell of the reference's smoothed-ball tumour (a cell whose value is
// not 0 when it has tissue): grid coordinates and the value in Real.
template <class Real>
struct BallCell {
    int x, y, z;
    Real value;
};

// The cells of the uniform bpd^3-block grid (MRAG level ceil(log2 bpd)) that
// lie in the smoothing band of the ball around tic, with their values, in
// the arithmetic of Glioma_ReactionDiffusion::_ic (Glioma/
// Glioma_ReactionDiffusion.cpp:155-164).  Returns false if a cell falls in
// the ball's core (psi < -1), which the reference's radius and width leave
// empty.
template <class Real>
bool ball_band_cells(int bpd, const double tic[3], std::vector<BallCell<Real>> &out);

}  // namespace gbfk_host
