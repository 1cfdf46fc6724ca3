// SPDX-License-Identifier: 0BSD
// ---------------------------------------------------------------------------
// Row strip of the global field with one halo row above and below: the I/O
// type of the CPU step task.  Same members and accessors as the reference's
// include/tile.hpp:10-33 (owned rows are 1..owned_rows(), row 0 and the last
// row are halos, storage row-major `nx` wide).
// ---------------------------------------------------------------------------
#pragma once
#include <vector>

namespace lpbf {

struct HaloTile {
    int idx = 0;
    int y0  = 0;           // first owned global row
    int y1  = 0;           // last owned global row (inclusive)
    int nx  = 0;

    int    step    = 0;
    double t       = 0.0;
    double x_laser = 0.0;
    double y_laser = 0.0;
    double q_scale = 1.0;  // 0 while the beam is off

    std::vector<double> data;

    int owned_rows() const noexcept { return y1 - y0 + 1; }
    int total_rows() const noexcept { return owned_rows() + 2; }
    double&       at(int r, int c)       noexcept { return data[r * nx + c]; }
    double        at(int r, int c) const noexcept { return data[r * nx + c]; }
};

}  // namespace lpbf
