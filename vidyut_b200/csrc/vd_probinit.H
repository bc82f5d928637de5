// amrex_probinit of the compiled-in case, fed the `prob.*` parameters of an
// inputs-file text.  A case written against this library's reader defines
// amrex_probinit(ProbParm&, vd::ParmParse&); a reference case directory
// compiled through the compatibility layer (VD_REFERENCE_CASE,
// vidyut_b200/compat) keeps the reference's amrex_probinit(ProbParm& host,
// ProbParm& device), which reads through amrex::ParmParse("prob") and
// copies the host struct into the device one: the library uploads the host
// struct itself afterwards.
#pragma once

#include "vd_parmparse.H"

inline void vd_probinit(ProbParm& h, const char* text)
{
    auto table = vd::ParmParse::parse(text ? text : "");
#ifdef VD_REFERENCE_CASE
    amrex::ParmParse::table() = &table;
    ProbParm d{};
    amrex_probinit(h, d);
    amrex::ParmParse::table() = nullptr;
#else
    vd::ParmParse pp(&table, "prob");
    amrex_probinit(h, pp);
#endif
}
