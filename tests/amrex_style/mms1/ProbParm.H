#ifndef MMS1_AMREX_PROBPARM_H
#define MMS1_AMREX_PROBPARM_H
#include <AMReX_REAL.H>

struct ProbParm
{
    int axdir = 0;
};
#endif
