// State-component indices after the species (Source/VarDefines.H:5-38), in
// terms of NUM_SPECIES, which the case's Chemistry.H defines.  Macros only,
// expanded where used, so this header may come before or after the case's
// Chemistry.H (a reference Chemistry.H includes VarDefines.H first).
#pragma once

#define EEN_ID (NUM_SPECIES)
#define ETEMP_ID (NUM_SPECIES + 1)
#define POT_ID (NUM_SPECIES + 2)
#define EFX_ID (NUM_SPECIES + 3)
#define EFY_ID (NUM_SPECIES + 4)
#define EFZ_ID (NUM_SPECIES + 5)
#define EJH_ID (NUM_SPECIES + 6)
#define EIH_ID (NUM_SPECIES + 7)
#define EEH_ID (NUM_SPECIES + 8)
#define REF_ID (NUM_SPECIES + 9)
#define SRFCH_ID (NUM_SPECIES + 10)
#define PHOTO_ION_SRC_ID (NUM_SPECIES + 11)
#define CMASK_ID (NUM_SPECIES + 12)
#define ECURX_ID (NUM_SPECIES + 13)
#define ECURY_ID (NUM_SPECIES + 14)
#define ECURZ_ID (NUM_SPECIES + 15)
#define ICURX_ID (NUM_SPECIES + 16)
#define ICURY_ID (NUM_SPECIES + 17)
#define ICURZ_ID (NUM_SPECIES + 18)
#define DCURX_ID (NUM_SPECIES + 19)
#define DCURY_ID (NUM_SPECIES + 20)
#define DCURZ_ID (NUM_SPECIES + 21)
#define NUM_PLASMAVARS (DCURZ_ID - NUM_SPECIES + 1)
#define NVAR (NUM_SPECIES + NUM_PLASMAVARS)
