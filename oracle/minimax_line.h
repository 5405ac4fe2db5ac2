/* minimax_line.h -- Chebyshev (minimax) straight-line fit shared by the oracle and the oracle
 * harness's LP stand-in.  TEST INFRASTRUCTURE ONLY.
 *
 * Given points (x_i, y_i) it returns the line y = a*x + b that minimises e = max_i |a x_i + b - y_i|,
 * i.e. the optimum of the 3-variable LP the reference solves per user
 * (src/include/alg/RegressionPruning/NormalLinearRegressionLP.hpp:181-213).  Method: the optimum
 * strip is bounded by lines parallel to an edge of the point set's upper or lower convex hull, so
 * every hull-edge slope is evaluated and the narrowest vertical strip is kept.  Arithmetic in double.
 */
#ifndef RKR_MINIMAX_LINE_H
#define RKR_MINIMAX_LINE_H
#ifdef __cplusplus
/* <cmath>, not <math.h>: in C++ libstdc++'s <math.h> exports the std:: float overloads (exp, ...)
 * into the global namespace, which would change the reference code compiled after it. */
#include <cmath>
#include <cstdlib>
#else
#include <math.h>
#include <stdlib.h>
#endif

static double mml_cross(const double *o, const double *a, const double *b) {
    return (a[0] - o[0]) * (b[1] - o[1]) - (a[1] - o[1]) * (b[0] - o[0]);
}
static int mml_cmp_pt(const void *pa, const void *pb) {
    const double *a = (const double *) pa, *b = (const double *) pb;
    if (a[0] != b[0]) return (a[0] > b[0]) - (a[0] < b[0]);
    return (a[1] > b[1]) - (a[1] < b[1]);
}
/* pts: n interleaved (x, y) pairs; reordered in place. */
static void minimax_line(double *pts, int n, double *a_out, double *b_out, double *e_out) {
    qsort(pts, (size_t) n, 2 * sizeof(double), mml_cmp_pt);
    double *lo = (double *) malloc(sizeof(double) * 2 * (size_t) (n > 0 ? n : 1));
    double *up = (double *) malloc(sizeof(double) * 2 * (size_t) (n > 0 ? n : 1));
    int nl = 0, nu = 0;
    for (int i = 0; i < n; i++) {
        while (nl >= 2 && mml_cross(lo + 2 * (nl - 2), lo + 2 * (nl - 1), pts + 2 * i) <= 0) nl--;
        lo[2 * nl] = pts[2 * i]; lo[2 * nl + 1] = pts[2 * i + 1]; nl++;
        while (nu >= 2 && mml_cross(up + 2 * (nu - 2), up + 2 * (nu - 1), pts + 2 * i) >= 0) nu--;
        up[2 * nu] = pts[2 * i]; up[2 * nu + 1] = pts[2 * i + 1]; nu++;
    }
    double best_e = INFINITY, best_a = 0, best_b = 0;
    for (int h = 0; h < 2; h++) {
        const double *hull = h ? up : lo;
        const int nh = h ? nu : nl;
        for (int k = 0; k + 1 < nh; k++) {
            const double dx = hull[2 * k + 2] - hull[2 * k];
            if (dx == 0) continue;
            const double a = (hull[2 * k + 3] - hull[2 * k + 1]) / dx;
            double mx = -INFINITY, mn = INFINITY;
            for (int i = 0; i < nu; i++) { const double r = up[2 * i + 1] - a * up[2 * i]; if (r > mx) mx = r; if (r < mn) mn = r; }
            for (int i = 0; i < nl; i++) { const double r = lo[2 * i + 1] - a * lo[2 * i]; if (r > mx) mx = r; if (r < mn) mn = r; }
            const double e = 0.5 * (mx - mn);
            if (e < best_e) { best_e = e; best_a = a; best_b = 0.5 * (mx + mn); }
        }
    }
    if (!(best_e < INFINITY)) {
        double mx = -INFINITY, mn = INFINITY;
        for (int i = 0; i < n; i++) { if (pts[2 * i + 1] > mx) mx = pts[2 * i + 1]; if (pts[2 * i + 1] < mn) mn = pts[2 * i + 1]; }
        best_a = 0; best_b = n > 0 ? 0.5 * (mx + mn) : 0; best_e = n > 0 ? 0.5 * (mx - mn) : 0;
    }
    free(lo); free(up);
    *a_out = best_a; *b_out = best_b; *e_out = best_e;
}
#endif
