// signal.cpp — crash-pulse signal processing on the host (C++17): the SAE
// J211 channel-frequency-class filter and linear resampling the reference
// applies to accelerometer histories (src/signal.rs). Histories are a few
// thousand samples; this is host work after a run.
#include <algorithm>
#include <cmath>
#include <vector>

#include "crush.h"
#include "errors.hpp"

namespace {

// One causal pass of the 2-pole low-pass over x, the signal padded at both
// ends by its point reflection about the end samples (`pad` samples each),
// returning the unpadded span (src/signal.rs:22-35).
void cfc_pass(const std::vector<double>& x, size_t pad, const double a[3], const double b[2], std::vector<double>& out) {
    const size_t n = x.size();
    std::vector<double> ext;
    ext.reserve(n + 2 * pad);
    for (size_t i = 0; i < pad; ++i) ext.push_back(2.0 * x[0] - x[pad - i]);
    ext.insert(ext.end(), x.begin(), x.end());
    for (size_t i = 1; i <= pad; ++i) ext.push_back(2.0 * x[n - 1] - x[n - 1 - i]);
    std::vector<double> y(ext.size(), 0.0);
    y[0] = ext[0];
    y[1] = ext[1];
    for (size_t i = 2; i < ext.size(); ++i) y[i] = a[0] * ext[i] + a[1] * ext[i - 1] + a[2] * ext[i - 2] + b[0] * y[i - 1] + b[1] * y[i - 2];
    out.assign(y.begin() + (long)pad, y.begin() + (long)(pad + n));
}

}  // namespace

extern "C" {

// cfc_filter, src/signal.rs:9-40: bilinear-transformed 2-pole Butterworth
// with the J211 prewarped corner (2.0775 x CFC), run forward then backward.
int crush_cfc_filter(const double* x, int64_t n, double dt, double cfc, double* y) {
    if (n < 0 || (n > 0 && (!x || !y))) return crush::fail(CRUSH_ERR_INVALID, "cfc filter: null signal or negative length");
    if (n < 4) {
        std::copy(x, x + n, y);
        return CRUSH_OK;
    }
    if (!(dt > 0.0) || !(cfc > 0.0)) return crush::fail(CRUSH_ERR_INVALID, "cfc filter: dt and cfc must be positive");
    const double wd = 2.0 * M_PI * cfc * 2.0775;
    const double half = wd * dt / 2.0;
    const double wa = std::sin(half) / std::cos(half);
    const double s2 = std::sqrt(2.0);
    const double den = 1.0 + s2 * wa + wa * wa;
    const double a0 = wa * wa / den;
    const double a[3] = {a0, 2.0 * a0, a0};
    const double b[2] = {-2.0 * (wa * wa - 1.0) / den, (-1.0 + s2 * wa - wa * wa) / den};
    // padding: ceil(3 / (cfc dt)) samples, at least 1 and at most n - 1
    const double want = std::ceil(3.0 / (cfc * dt));
    size_t pad = want >= 1.8e19 ? ~(size_t)0 : (want > 0.0 ? (size_t)want : 0);  // a saturating float-to-size cast
    pad = std::max<size_t>(std::min<size_t>(pad, (size_t)n - 1), 1);
    std::vector<double> in(x, x + n), fwd, back;
    cfc_pass(in, pad, a, b, fwd);
    std::reverse(fwd.begin(), fwd.end());
    cfc_pass(fwd, pad, a, b, back);
    std::reverse(back.begin(), back.end());
    std::copy(back.begin(), back.end(), y);
    return CRUSH_OK;
}

// resample, src/signal.rs:42-66: for each grid time, the segment of (t, y)
// that holds it (held at the ends), linearly interpolated.
int crush_resample(const double* t, const double* y, int64_t n, double t0, double dt, double t_end, double* tu, double* yu,
                   int64_t cap, int64_t* n_out) {
    if (!t || !y || n < 1 || !n_out || cap < 0 || (cap > 0 && (!tu || !yu)))
        return crush::fail(CRUSH_ERR_INVALID, "resample: need at least one sample and output buffers");
    if (!(dt > 0.0)) return crush::fail(CRUSH_ERR_INVALID, "resample: dt must be positive");
    const double span = std::floor((t_end - t0) / dt);
    const int64_t m = span >= 0.0 ? (int64_t)span + 1 : 1;  // the reference's usize cast floors negatives at 0
    *n_out = m;
    size_t j = 0;
    const size_t len = (size_t)n;
    for (int64_t k = 0; k < m && k < cap; ++k) {
        const double tk = t0 + (double)k * dt;
        while (j + 1 < len && t[j + 1] < tk) ++j;
        double v;
        if (j + 1 >= len) v = y[len - 1];
        else if (tk <= t[0]) v = y[0];
        else {
            const double w = (tk - t[j]) / (t[j + 1] - t[j]);
            v = y[j] + w * (y[j + 1] - y[j]);
        }
        tu[k] = tk;
        yu[k] = v;
    }
    return CRUSH_OK;
}

}  // extern "C"
