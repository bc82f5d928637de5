#pragma once
#include "vd_defs.H"

// electrode layout of the user potential callback (UserFunctions.H), in
// units of the cube's edge and volts
struct ProbParm
{
    vd::Real trode_rad = 0.125;
    vd::Real trode_sep = 0.25;
    vd::Real trode_volt = 60.0;
    vd::Real subs_rad = 0.25;
};
