#pragma once
#include "vd_defs.H"

struct ProbParm
{
    int unused = 0;
};
