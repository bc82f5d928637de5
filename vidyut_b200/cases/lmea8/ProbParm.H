// Problem parameters of the LMEA case: uniform initial densities per species
// (the benchmark overwrites them with a seeded field through vd_set_state),
// electron temperature 1 eV.
#pragma once
#include "vd_defs.H"

struct ProbParm
{
    vd::Real n0[8] = {1e16, 4e15, 3e15, 2e15, 2e15, 1e15, 2.45e25, 1e14};
    vd::Real te = 11604.518;
};
