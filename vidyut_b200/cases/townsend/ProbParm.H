// Problem parameters of the Townsend discharge case: a uniform background
// plus up to VD_MAX_BLOBS Gaussian electron/ion blobs
// n = bg + sum_b ampl_b exp(-|x - c_b|^2 / (2 sigma_b^2)), ions = electrons,
// the same kind of seeded multi-blob start as test/models/Streamer3d/Prob.H:64-125.
#pragma once
#include "vd_defs.H"

#define VD_MAX_BLOBS 8

struct ProbParm
{
    vd::Real bg = 1.0e13;
    vd::Real ngas = 2.45e25;
    vd::Real te = 5802.25;
    int nblobs = 0;
    vd::Real cx[VD_MAX_BLOBS] = {0};
    vd::Real cy[VD_MAX_BLOBS] = {0};
    vd::Real cz[VD_MAX_BLOBS] = {0};
    vd::Real ampl[VD_MAX_BLOBS] = {0};
    vd::Real sigma[VD_MAX_BLOBS] = {0};
    int twod = 0;
};
