#pragma once
#include "vd_defs.H"

struct ProbParm
{
    int axdir = 0;
};
