// The reference's mixed-precision propagator (Fprop_alt_Standard_eo_Richardson:
// FP64 Richardson outer loop, APrecond_Mixedprec, FP32 inner CG,
// src/lib_alt/Measurements/Fermion/fprop_alt_Standard_eo_Richardson-tmpl.h)
// over AField<double|float, B200>, instantiated as the Accel build does
// (src/lib_alt_Accel/Measurements/Fermion/fprop_alt_Standard_eo_Richardson.cpp).
// Its smeared-operator branch needs AFopr_Smeared_alt and Director_alt_Smear
// for the B200 field, instantiated here from the reference's templates; the
// smearing itself stays the reference's host Field_G path.
#define DIRECTOR_ALT_SMEARED_IMPLEMENTED
#include "lib_alt_B200/Field/afield.h"

#include "lib/Fopr/afopr_Smeared_alt.h"
#include "lib/Fopr/afopr_Smeared_alt-tmpl.h"
#include "lib/ResourceManager/threadManager.h"
#include "lib_alt/Smear/director_alt_Smear.h"
#include "lib_alt/Smear/director_alt_Smear-tmpl.h"
#include "lib_alt/Solver/aprecond_Mixedprec.h"
#include "lib_alt/Solver/asolver_Richardson.h"
#include "lib_alt/Measurements/Fermion/fprop_alt_Standard_eo_Richardson.h"
#include "lib_alt/Measurements/Fermion/fprop_alt_Standard_eo_Richardson-tmpl.h"

template class Director_alt_Smear<AField<double, B200> >;
template class AFopr_Smeared_alt<AField<double, B200> >;

template<>
const std::string Fprop_alt_Standard_eo_Richardson<AField<double, B200>, AField<float, B200> >::class_name
  = "Fprop_alt_Standard_eo_Richardson<AField<double,B200>, AField<float,B200> >";
template class Fprop_alt_Standard_eo_Richardson<AField<double, B200>, AField<float, B200> >;
