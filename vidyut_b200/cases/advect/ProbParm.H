#pragma once
#include "vd_defs.H"

struct ProbParm
{
    int one_dim = 1;
    vd::Real blobrad = 0.1;
    vd::Real velx = 1.0;
    vd::Real vely = 0.0;
    vd::Real velz = 0.0;
};
