#include "Chemistry.H"

void CKSYMS_STR(amrex::Vector<std::string>& kname)
{
    kname.resize(NUM_SPECIES);
    kname[E_ID] = "E";
    kname[NI_ID] = "NI";
}
