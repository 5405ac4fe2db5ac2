// LP stand-in for the oracle harness.  The reference calls sdlp::linprog<3> only with the LP of
// NormalLinearRegressionLP::LinearProgram (NormalLinearRegressionLP.hpp:181-213): minimise e over
// (a, b, e) subject to rows s*(x a + b) - e <= s*y, s = +-1, i.e. a minimax line through the points
// (x, y).  This stand-in recovers the points from the rows and solves that problem exactly with
// the oracle's own minimax_line (oracle/minimax_line.h); it is not a general LP solver.
#pragma once
#include <vector>
extern "C" {
#include "../../../minimax_line.h"
}
namespace sdlp {
template <int d, typename C, typename A, typename B, typename X>
inline float linprog(const C &, const A &Am, const B &b, const int *, X &x) {
    std::vector<double> pts;
    pts.reserve((size_t) Am.rows());
    for (long i = 0; i < Am.rows(); i++) {
        const double s = Am(i, 1);  // +1 or -1
        if (s == 0) continue;
        const double px = Am(i, 0) * s, py = b(i) * s;
        bool dup = false;
        const size_t n = pts.size() / 2;
        if (n > 0 && pts[2 * n - 2] == px && pts[2 * n - 1] == py) dup = true;
        if (!dup) { pts.push_back(px); pts.push_back(py); }
    }
    double a = 0, bb = 0, e = -1;
    if (!pts.empty()) minimax_line(pts.data(), (int) (pts.size() / 2), &a, &bb, &e);
    x[0] = (float) a; x[1] = (float) bb; x[2] = (float) e;
    return (float) e;
}
}  // namespace sdlp
