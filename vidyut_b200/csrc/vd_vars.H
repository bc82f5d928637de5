// State-component indices of one Vidyut cell, after Source/VarDefines.H:5-38.
// The species come first (0 .. NUM_SPECIES-1, defined by the case's
// Chemistry.H), then the plasma variables.  Storage is one FP64 array per
// component (structure of arrays, x fastest), the layout of an AMReX
// MultiFab box.
#pragma once

#include "vd_defs.H"
#include "vd_ids.H"
#include <Chemistry.H>


#include <ProbParm.H>
