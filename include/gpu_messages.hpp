// SPDX-License-Identifier: 0BSD
// ---------------------------------------------------------------------------
// Messages on the edges of the GPU step graph.  Member names, order and types
// match the reference's include/gpu_messages.hpp:18-50 (Tick is 56 bytes with
// `wrapped` at 48 and `dump` at 49), so plans built by reference drivers can
// be handed to this library as raw arrays.
// ---------------------------------------------------------------------------
#pragma once
#include <memory>
#include <vector>

namespace lpbf {

// One time step of the laser plan.  x_l/y_l/q_scale are the values the step
// kernel uses for step `step`; x_laser_csv/wrapped are the post-advance laser
// state that the metrics use; dump marks snapshot/csv steps.
struct Tick {
    int    step;
    double t;
    double x_l, y_l;
    double q_scale;
    double x_laser_csv;
    bool   wrapped;
    bool   dump;
};
static_assert(sizeof(Tick) == 56, "Tick ABI");

struct MetricsMsg {
    int    step;
    double t;
    double x_laser_csv;
    bool   wrapped;
    bool   dump;
    double tmax;
    int    x_hot;
    int    ymin, ymax;
    std::vector<double> hot_col;   // T along column x_hot (empty if unused)
};

struct SnapshotMsg {
    int step;
    std::shared_ptr<std::vector<double>> field;   // nx*ny row-major
};

struct StepResult { int step; };

}  // namespace lpbf
