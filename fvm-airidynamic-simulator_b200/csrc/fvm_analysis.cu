// fvm_analysis.cu -- host-side analysis of force-coefficient histories
// (C ABI fvm_shedding_stats).  No reference counterpart: the reference prints
// no drag or lift; the Strouhal number of a vortex street is read off the lift
// history here.
//
// Method: the lift coefficient minus its mean over the window crosses zero
// upward once per shedding cycle.  Crossing times are located by linear
// interpolation between samples; the period is the span between the first
// and last crossing over the number of whole cycles in it, and the mean drag
// and lift statistics are integrated (trapezoids over the piecewise-linear
// history) over exactly that span, so a partial cycle at either end does not
// bias them.
#include <cmath>
#include <vector>

#include "fvm_handle.h"

// Integral of the piecewise-linear function through (t[k], f[k]) over [a, b]
// (a, b inside [t[0], t[n-1]]); g applied to the interpolated values.
template <class G>
static double integrate(const double *t, const double *f, int n, double a, double b, G g) {
    double acc = 0.0;
    for (int k = 0; k + 1 < n; k++) {
        const double lo = std::fmax(a, t[k]), hi = std::fmin(b, t[k + 1]);
        if (hi <= lo) continue;
        const double h = t[k + 1] - t[k];
        const double fl = f[k] + (f[k + 1] - f[k]) * (lo - t[k]) / h;
        const double fh = f[k] + (f[k + 1] - f[k]) * (hi - t[k]) / h;
        // Simpson on the linear piece keeps g(f) exact for quadratic g
        const double fm = 0.5 * (fl + fh);
        acc += (hi - lo) * (g(fl) + 4.0 * g(fm) + g(fh)) / 6.0;
    }
    return acc;
}

extern "C" int fvm_shedding_stats(const double *t, const double *cd, const double *cl, int n, double ref_length,
                                  double u_inf, fvm_shedding *out) {
    if (!t || !cd || !cl || !out) return fvm_internal_set_error(FVM_ERR_INVALID, "fvm_shedding_stats: null pointer");
    if (n < 3 || !(ref_length > 0.0) || !(u_inf > 0.0))
        return fvm_internal_set_error(FVM_ERR_INVALID,
                                      "fvm_shedding_stats: need n >= 3 samples and positive ref_length, u_inf");
    for (int k = 0; k + 1 < n; k++)
        if (!(t[k + 1] > t[k]))
            return fvm_internal_set_error(FVM_ERR_INVALID, "fvm_shedding_stats: times must increase strictly");
    double mean = 0.0;
    for (int k = 0; k < n; k++) mean += cl[k];
    mean /= n;
    std::vector<double> cross;
    for (int k = 0; k + 1 < n; k++) {
        const double a = cl[k] - mean, b = cl[k + 1] - mean;
        if (a < 0.0 && b >= 0.0) cross.push_back(t[k] + (t[k + 1] - t[k]) * (-a) / (b - a));
    }
    if (cross.size() < 2)
        return fvm_internal_set_error(FVM_ERR_INVALID,
                                      "fvm_shedding_stats: the lift history holds less than one shedding cycle");
    const double a = cross.front(), b = cross.back();
    const int cycles = (int)cross.size() - 1;
    const double span = b - a;
    out->cycles = cycles;
    out->period = span / cycles;
    out->strouhal = ref_length / (out->period * u_inf);
    out->cd_mean = integrate(t, cd, n, a, b, [](double x) { return x; }) / span;
    out->cl_mean = integrate(t, cl, n, a, b, [](double x) { return x; }) / span;
    const double m = out->cl_mean;
    out->cl_rms = std::sqrt(std::fmax(0.0, integrate(t, cl, n, a, b, [m](double x) { return (x - m) * (x - m); }) / span));
    out->reserved = 0;
    return FVM_OK;
}
