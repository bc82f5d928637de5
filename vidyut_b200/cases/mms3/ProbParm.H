#pragma once
#include "vd_defs.H"

struct ProbParm
{
    int axdir = 0;
    vd::Real n0 = 1e6;
};
