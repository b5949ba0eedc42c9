// ref_ice_harness.cpp -- driver over the REFERENCE ice optical constants
// (hex_atlas/src/ice_optics.cpp, compiled from its source by oracle/build_ref.sh).  Test
// infrastructure only: it generates the golden values the library's ice index is pinned to.
//
// stdin: one vacuum wavelength in nm per line.  stdout per line: "ok n kappa lower_nm upper_nm
// fraction" in hexadecimal floating point (exact), or "invalid" / "error" for the reference's
// std::invalid_argument / other exceptions.
#include <ice_crystal/ice_optics.hpp>

#include <cstdio>
#include <iostream>
#include <stdexcept>
#include <string>

int main()
{
    std::string line;
    while (std::getline(std::cin, line)) {
        if (line.empty()) continue;
        const double nm = std::stod(line);
        try {
            const auto s = iceCrystal::optics::evaluate_ice_wb2008(nm);
            std::printf("ok %a %a %a %a %a\n", s.n, s.kappa, s.lower_nm, s.upper_nm, s.log_wavelength_fraction);
        } catch (const std::invalid_argument&) {
            std::printf("invalid\n");
        } catch (const std::exception&) {
            std::printf("error\n");
        }
    }
    return 0;
}
