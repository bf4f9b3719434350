// Host-side Gauss-Legendre rules and Gauss-order thresholds for the device
// fill kernels.  Same construction as the reference's inductance/gauss.rs:
// Newton iteration on the three-term Legendre recurrence from the
// cos(pi (k + 3/4) / (n + 1/2)) initial guess, weights 2 / ((1 - x^2) P'^2),
// and thresholds sinh(ln(1/tol) / 2n) (gauss.rs:100-118).  Compiled with
// -ffp-contract=off so that nodes and thresholds equal the reference's bits.
#include <cmath>
#include <limits>

#include "fh_device.cuh"

namespace fhb {

namespace {

void legendre_rule(int n, double *nodes, double *weights) {
    const double pi = 3.14159265358979323846;
    const double eps = std::numeric_limits<double>::epsilon();
    const double nf = (double)n;
    auto eval = [&](double x, double &p_prev, double &p) {
        p_prev = 1.0;
        p = x;
        for (int j = 1; j < n; ++j) {
            double jf = (double)j;
            double next = ((2.0 * jf + 1.0) * x * p - jf * p_prev) / (jf + 1.0);
            p_prev = p;
            p = next;
        }
    };
    for (int k = 0; k < (n + 1) / 2; ++k) {
        double x = std::cos(pi * ((double)k + 0.75) / (nf + 0.5));
        double deriv = 1.0;
        for (int it = 0; it < 100; ++it) {
            double pp, p;
            eval(x, pp, p);
            deriv = nf * (x * p - pp) / (x * x - 1.0);
            double step = p / deriv;
            x -= step;
            double ax = std::fabs(x);
            if (std::fabs(step) <= 4.0 * eps * (ax > 1e-3 ? ax : 1e-3)) break;
        }
        if (n % 2 == 1 && k == n / 2) {
            x = 0.0;
            double pp, p;
            eval(x, pp, p);
            deriv = nf * (x * p - pp) / (x * x - 1.0);
        }
        double w = 2.0 / ((1.0 - x * x) * deriv * deriv);
        nodes[n - 1 - k] = x;
        nodes[k] = -x;
        weights[n - 1 - k] = w;
        weights[k] = w;
    }
}

}  // namespace

void gauss_rule(int n, double *nodes, double *weights) { legendre_rule(n, nodes, weights); }

void host_quad_tables(QuadTables &t) {
    for (int n = 0; n <= kMaxRule; ++n)
        for (int k = 0; k < kMaxRule; ++k) t.nodes[n][k] = t.weights[n][k] = 0.0;
    for (int n = 1; n <= kMaxRule; ++n) legendre_rule(n, t.nodes[n], t.weights[n]);
    const double lp = std::log(1.0 / 1e-8), ls = std::log(1.0 / 1e-6);
    for (int n = 1; n <= 16; ++n) t.point_thresholds[n - 1] = std::sinh(lp / (2.0 * (double)n));
    for (int n = 1; n <= 8; ++n) t.sample_thresholds[n - 1] = std::sinh(ls / (2.0 * (double)n));
}

}  // namespace fhb
