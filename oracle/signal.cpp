// signal.cpp — TEST INFRASTRUCTURE ONLY (see oracle.hpp).
// Restates src/signal.rs:9-40 (cfc_filter) and :42-66 (resample) as written:
// the checker for the library's crush_cfc_filter / crush_resample.
#include <cmath>

#include "oracle.hpp"

namespace oracle {

// cfc_filter, src/signal.rs:9-40.
std::vector<double> cfc_filter(const std::vector<double>& x, double dt, double cfc) {
    if (x.size() < 4) return x;
    const double wd = 2.0 * M_PI * cfc * 2.0775;
    const double wa = std::sin(wd * dt / 2.0) / std::cos(wd * dt / 2.0);
    const double s2 = std::sqrt(2.0);
    const double den = 1.0 + s2 * wa + wa * wa;
    const double a0 = wa * wa / den;
    const double a1 = 2.0 * a0;
    const double a2 = a0;
    const double b1 = -2.0 * (wa * wa - 1.0) / den;
    const double b2 = (-1.0 + s2 * wa - wa * wa) / den;
    auto pass = [&](const std::vector<double>& in) {
        const size_t n = in.size();
        const double p = std::ceil(3.0 / (cfc * dt));
        size_t pad = p >= 1.8e19 ? ~(size_t)0 : (p > 0.0 ? (size_t)p : 0);  // `as usize` saturates
        pad = std::max<size_t>(std::min<size_t>(pad, n - 1), 1);
        std::vector<double> ext;
        for (size_t i = 0; i < pad; ++i) ext.push_back(2.0 * in[0] - in[pad - i]);
        for (double v : in) ext.push_back(v);
        for (size_t i = 1; i <= pad; ++i) ext.push_back(2.0 * in[n - 1] - in[n - 1 - i]);
        std::vector<double> y(ext.size(), 0.0);
        y[0] = ext[0];
        y[1] = ext[1];
        for (size_t i = 2; i < ext.size(); ++i) y[i] = a0 * ext[i] + a1 * ext[i - 1] + a2 * ext[i - 2] + b1 * y[i - 1] + b2 * y[i - 2];
        return std::vector<double>(y.begin() + (long)pad, y.begin() + (long)(pad + n));
    };
    std::vector<double> fwd = pass(x);
    std::vector<double> rev(fwd.rbegin(), fwd.rend());
    rev = pass(rev);
    return std::vector<double>(rev.rbegin(), rev.rend());
}

// resample, src/signal.rs:42-66.
void resample(const std::vector<double>& t, const std::vector<double>& y, double t0, double dt, double t_end, std::vector<double>* tu,
              std::vector<double>* yu) {
    const double f = std::floor((t_end - t0) / dt);
    const size_t n = (f > 0.0 ? (size_t)f : 0) + 1;
    tu->clear();
    yu->clear();
    size_t j = 0;
    for (size_t k = 0; k < n; ++k) {
        const double tk = t0 + (double)k * dt;
        while (j + 1 < t.size() && t[j + 1] < tk) ++j;
        double v;
        if (j + 1 >= t.size()) v = y[t.size() - 1];
        else if (tk <= t[0]) v = y[0];
        else {
            const double w = (tk - t[j]) / (t[j + 1] - t[j]);
            v = y[j] + w * (y[j + 1] - y[j]);
        }
        tu->push_back(tk);
        yu->push_back(v);
    }
}

}  // namespace oracle
