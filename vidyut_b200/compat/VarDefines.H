// Stand-in for the AMReX / reference header of this name: see vd_amrex_compat.H.
#pragma once
#include "vd_amrex_compat.H"
