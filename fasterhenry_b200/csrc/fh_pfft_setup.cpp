// Host part of the precorrected-FFT set-up: parameters and the grid, by the
// reference's method (pfft/mod.rs:332-460, grid.rs:44-95): spacing h over the
// filaments' bounding box, padded by half a stencil, h from GridSpacing::Auto
// (about cells_per_filament cells per filament) or fixed; the near-field
// radius k h.  The near pairs (fh_near.cu), the projections and the grid
// approximations of the near pairs (fh_pfft_setup.cu) are built on the
// device.
#include <algorithm>
#include <cmath>
#include <limits>

#include "fh_pfft.h"

namespace fhb {

int64_t smooth_size(int64_t n) {
    int64_t m = std::max<int64_t>(n, 1);
    for (;; ++m) {
        int64_t r = m;
        for (int p : {2, 3, 5})
            while (r % p == 0) r /= p;
        if (r == 1) return m;
    }
}

double auto_spacing(const double extent[3], double cells) {
    const double largest = std::max(extent[0], std::max(extent[1], extent[2]));
    auto count = [&](double h) {
        double c = 1.0;
        for (int a = 0; a < 3; ++a) c *= std::max(extent[a] / h, 1.0);
        return c;
    };
    if (cells <= 1.0 || largest <= 0.0) return std::max(largest, std::numeric_limits<double>::min());
    double small = largest / cells, large = largest;
    for (int it = 0; it < 200; ++it) {
        const double mid = std::sqrt(small * large);
        if (count(mid) > cells)
            small = mid;
        else
            large = mid;
    }
    return large;
}

fh_status pfft_setup(const fh_filament *fil, int64_t n, const PfftConfig &cfg, PfftSetup &out, fh_error_info *err) {
    if (cfg.order < 1) return fail(err, FH_ERR_PFFT, "invalid pFFT parameter: interpolation_order must be at least 1");
    if (!(std::isfinite(cfg.near_field_radius) && cfg.near_field_radius >= (double)(cfg.order + 1)))
        return fail(err, FH_ERR_PFFT,
                    "invalid pFFT parameter: near_field_radius must be finite and at least interpolation_order + 1");
    if (cfg.order > 15) return fail(err, FH_ERR_PFFT, "invalid pFFT parameter: interpolation_order above 15");
    if (!cfg.fixed_spacing && !(cfg.cells_per_filament > 0.0 && std::isfinite(cfg.cells_per_filament)))
        return fail(err, FH_ERR_PFFT, "invalid pFFT parameter: cells_per_filament must be positive and finite");
    if (cfg.fixed_spacing && !(cfg.spacing > 0.0 && std::isfinite(cfg.spacing)))
        return fail(err, FH_ERR_PFFT, "invalid pFFT parameter: grid spacing must be positive and finite");
    out = PfftSetup();
    out.n = n;
    if (n == 0) return FH_OK;

    // Bounding box of the filaments' volumes (pfft/mod.rs:600-611).
    double lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
        lo[a] = std::numeric_limits<double>::infinity();
        hi[a] = -std::numeric_limits<double>::infinity();
    }
    for (int64_t i = 0; i < n; ++i) {
        const fh_filament &f = fil[i];
        for (int a = 0; a < 3; ++a) {
            const double reach = 0.5 * (f.width * std::fabs(f.dir_width[a]) + f.height * std::fabs(f.dir_height[a]));
            lo[a] = std::min(lo[a], std::min(f.start[a] - reach, f.end[a] - reach));
            hi[a] = std::max(hi[a], std::max(f.start[a] + reach, f.end[a] + reach));
        }
    }
    double extent[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
    const double h = cfg.fixed_spacing ? cfg.spacing : auto_spacing(extent, cfg.cells_per_filament * (double)n);
    PfftGrid &g = out.grid;
    g.spacing = h;
    g.stencil = cfg.order + 1;
    const double pad = (double)((g.stencil + 1) / 2);
    for (int a = 0; a < 3; ++a) {
        g.origin[a] = lo[a] - pad * h;
        const double span = (hi[a] - g.origin[a]) / h;
        g.dims[a] = (int64_t)std::floor(span + 0.5 * g.stencil) + 2;
        out.padded[a] = padded_size(g.dims[a]);
    }
    const double padded_pts = (double)out.padded[0] * (double)out.padded[1] * (double)out.padded[2];
    if (padded_pts > (double)kMaxFftPoints || (double)g.len() > 4294967295.0)
        return fail(err, FH_ERR_PFFT,
                    "pFFT grid of " + std::to_string((long long)padded_pts) + " padded points exceeds the limit of " +
                        std::to_string((long long)kMaxFftPoints));
    out.radius = cfg.near_field_radius * h;
    out.directions.resize((size_t)n * 3);
    for (int64_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) out.directions[3 * i + a] = fil[i].dir_length[a];
    for (int a = 0; a < 3; ++a) {
        bool any = false;
        for (int64_t i = 0; i < n && !any; ++i) any = fil[i].dir_length[a] != 0.0;
        if (any) out.components.push_back(a);
    }
    return FH_OK;
}

}  // namespace fhb
