// common.hpp — shared host-side helpers: error reporting, constants.
#pragma once
#include <cstdarg>
#include <cstdio>
#include <string>

#include "../../../include/edus_b200.h"

namespace edus {

// headers/Constants.h:14-36 of the reference (a.u. conversions).
constexpr double kPi = 3.14159265358979323846;
constexpr double kC = 137.036;
constexpr double kTimeAuFs = 0.02418884326505;
constexpr double kTimeFsAu = 1.0 / 0.02418884326505;
constexpr double kEnergyAuEv = 27.211396;
constexpr double kEnergyEvAu = 1.0 / 27.211396;
constexpr double kSpaceAuA = 0.52917721092;
constexpr double kSpaceAAu = 1.0 / 0.52917721092;
constexpr double kIntensityAuWcm2 = 3.50944758e+16;
constexpr double kLaserIntensityConst = 3.51e+16;  // headers/Laser.h:29-31 uses this, not the exact value

// Records the message of the last failure for edus_last_error() and returns code.
int fail(int code, const char* fmt, ...);
void clear_error();

}  // namespace edus
