// icp_ice_optics.hpp -- refractive index of ice Ih for the prism records: the compilation of
// Warren & Brandt (2008), J. Geophys. Res. 113, D14220, DOI 10.1029/2007JD009744 (author table
// IOP_2008_ASCIItable.dat), restricted to 199..1100 nm.  The same published rows are what the
// reference interpolates (hex_atlas/src/ice_optics.cpp:13-30), so the index of a record agrees bit
// for bit.  Host code only, binary64.
//
// Between two table wavelengths a < lambda < b the real index is linear and the imaginary index
// log-linear in log(lambda):  f = ln(lambda / a) / ln(b / a),  n = n_a + f (n_b - n_a),
// kappa = exp(ln kappa_a + f (ln kappa_b - ln kappa_a)).  At a table wavelength the row is
// returned as it is.  Supported: 200 <= lambda <= 1100 nm, no extrapolation.
#pragma once
#include <cmath>
#include <cstddef>

namespace icp::host {

struct IceRow {
    double nm, n, kappa; // vacuum wavelength (nm), real index, imaginary index
};

// Warren & Brandt (2008), vacuum wavelength in nm, ascending.
inline constexpr IceRow kIceWB2008[] = {
    {199, 1.3943, 9.565E-011},
    {201, 1.3914, 3.249E-011},
    {201.9, 1.3901, 2.000E-011},
    {210, 1.3801, 2.000E-011},
    {250, 1.3509, 2.000E-011},
    {300, 1.3339, 2.000E-011},
    {350, 1.3249, 2.000E-011},
    {390, 1.3203, 2.000E-011},
    {400, 1.3194, 2.365E-011},
    {410, 1.3185, 2.669E-011},
    {420, 1.3177, 3.135E-011},
    {430, 1.3170, 4.140E-011},
    {440, 1.3163, 6.268E-011},
    {450, 1.3157, 9.239E-011},
    {460, 1.3151, 1.325E-010},
    {470, 1.3145, 1.956E-010},
    {480, 1.3140, 2.861E-010},
    {490, 1.3135, 4.172E-010},
    {500, 1.3130, 5.889E-010},
    {510, 1.3126, 8.036E-010},
    {520, 1.3121, 1.076E-009},
    {530, 1.3117, 1.409E-009},
    {540, 1.3114, 1.813E-009},
    {550, 1.3110, 2.289E-009},
    {560, 1.3106, 2.839E-009},
    {570, 1.3103, 3.461E-009},
    {580, 1.3100, 4.159E-009},
    {590, 1.3097, 4.930E-009},
    {600, 1.3094, 5.730E-009},
    {610, 1.3091, 6.890E-009},
    {620, 1.3088, 8.580E-009},
    {630, 1.3085, 1.040E-008},
    {640, 1.3083, 1.220E-008},
    {650, 1.3080, 1.430E-008},
    {660, 1.3078, 1.660E-008},
    {670, 1.3076, 1.890E-008},
    {680, 1.3073, 2.090E-008},
    {690, 1.3071, 2.400E-008},
    {700, 1.3069, 2.900E-008},
    {710, 1.3067, 3.440E-008},
    {720, 1.3065, 4.030E-008},
    {730, 1.3062, 4.300E-008},
    {740, 1.3060, 4.920E-008},
    {750, 1.3059, 5.870E-008},
    {760, 1.3057, 7.080E-008},
    {770, 1.3055, 8.580E-008},
    {780, 1.3053, 1.020E-007},
    {790, 1.3051, 1.180E-007},
    {800, 1.3049, 1.340E-007},
    {810, 1.3047, 1.400E-007},
    {820, 1.3046, 1.430E-007},
    {830, 1.3044, 1.450E-007},
    {840, 1.3042, 1.510E-007},
    {850, 1.3040, 1.830E-007},
    {860, 1.3039, 2.150E-007},
    {870, 1.3037, 2.650E-007},
    {880, 1.3035, 3.350E-007},
    {890, 1.3033, 3.920E-007},
    {900, 1.3032, 4.200E-007},
    {910, 1.3030, 4.440E-007},
    {920, 1.3028, 4.740E-007},
    {930, 1.3027, 5.110E-007},
    {940, 1.3025, 5.530E-007},
    {950, 1.3023, 6.020E-007},
    {960, 1.3022, 7.550E-007},
    {970, 1.3020, 9.260E-007},
    {980, 1.3019, 1.120E-006},
    {990, 1.3017, 1.330E-006},
    {1000, 1.3015, 1.620E-006},
    {1010, 1.3014, 2.000E-006},
    {1020, 1.3012, 2.250E-006},
    {1030, 1.3010, 2.330E-006},
    {1040, 1.3009, 2.330E-006},
    {1050, 1.3007, 2.170E-006},
    {1060, 1.3005, 1.960E-006},
    {1070, 1.3003, 1.810E-006},
    {1080, 1.3002, 1.740E-006},
    {1090, 1.3000, 1.730E-006},
    {1100, 1.2998, 1.700E-006}
};

struct IceIndex {
    double n, kappa, lower_nm, upper_nm, fraction;
};

// false outside 200..1100 nm (or for a non-finite wavelength)
inline bool ice_index_wb2008(double nm, IceIndex& out)
{
    if (!std::isfinite(nm) || nm < 200.0 || nm > 1100.0) return false;
    constexpr std::size_t rows = sizeof(kIceWB2008) / sizeof(kIceWB2008[0]);
    std::size_t lo = 0, hi = rows; // first row with a wavelength not below nm
    while (lo < hi) {
        const std::size_t mid = lo + (hi - lo) / 2;
        if (kIceWB2008[mid].nm < nm) lo = mid + 1;
        else hi = mid;
    }
    if (lo == rows || lo == 0) return false; // 200..1100 lies inside the table; not reached
    const IceRow& b = kIceWB2008[lo];
    if (b.nm == nm) {
        out = {b.n, b.kappa, b.nm, b.nm, 0.0};
        return true;
    }
    const IceRow& a = kIceWB2008[lo - 1];
    const double f = std::log(nm / a.nm) / std::log(b.nm / a.nm);
    const double n = a.n + f * (b.n - a.n);
    const double kappa = std::exp(std::log(a.kappa) + f * (std::log(b.kappa) - std::log(a.kappa)));
    out = {n, kappa, a.nm, b.nm, f};
    return n > 0 && kappa > 0 && std::isfinite(n) && std::isfinite(kappa);
}

} // namespace icp::host
