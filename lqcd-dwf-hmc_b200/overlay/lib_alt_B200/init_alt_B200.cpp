// Device selection, factory registration and the instantiations of the
// reference's own alt templates over AField<REAL, B200>: the counterpart of
// the Accel build's init_alt_Accel.cpp (src/lib_alt_Accel/init_alt_Accel.cpp:
// 20-49), bridge_init_factory_alt_Accel.cpp and Solver/*.cpp.  The template
// bodies compiled here are the reference's (asolver_CG-tmpl.h,
// asolver_Richardson-tmpl.h, aprecond_Mixedprec-tmpl.h,
// ashiftsolver_CG-tmpl.h); only the field and the operator are this
// library's.
#include "lib_alt_B200/Field/afield.h"
#include "lib_alt_B200/Fopr/afopr_Domainwall_5din_eo.h"
#include "lib_alt_B200/init_alt_B200.h"

#include "lib/Fopr/afopr.h"
#include "lib/ResourceManager/threadManager.h"
#include "lib_alt/Solver/asolver.h"
#include "lib_alt/Solver/asolver_CG.h"
#include "lib_alt/Solver/asolver_CG-tmpl.h"
#include "lib_alt/Solver/asolver_Richardson.h"
#include "lib_alt/Solver/asolver_Richardson-tmpl.h"
#include "lib_alt/Solver/aprecond_Mixedprec.h"
#include "lib_alt/Solver/aprecond_Mixedprec-tmpl.h"
#include "lib/Solver/ashiftsolver_CG.h"
#include "lib/Solver/ashiftsolver_CG-tmpl.h"

typedef AField<double, B200> AFIELD_d;
typedef AField<float, B200>  AFIELD_f;

template<>
const std::string ASolver_CG<AFIELD_d>::class_name = "ASolver_CG<AField<double,B200> >";
template<>
const std::string ASolver_CG<AFIELD_f>::class_name = "ASolver_CG<AField<float,B200> >";
template class ASolver_CG<AFIELD_d>;
template class ASolver_CG<AFIELD_f>;

template class ASolver_Richardson<AFIELD_d>;
template class APrecond_Mixedprec<AFIELD_d, AFIELD_f>;
template class AShiftsolver_CG<AFIELD_d, AFopr<AFIELD_d> >;

template<typename AFIELD>
bool ASolver<AFIELD>::init_factory()
{
  return ASolver_CG<AFIELD>::register_factory();
}

template class ASolver<AFIELD_d>;
template class ASolver<AFIELD_f>;

template<>
bool AFopr<AFIELD_d>::init_factory()
{
  return AFopr_Domainwall_5din_eo<AFIELD_d>::register_factory();
}

template<>
bool AFopr<AFIELD_f>::init_factory()
{
  return AFopr_Domainwall_5din_eo<AFIELD_f>::register_factory();
}

bool init_alt_B200(int rank, int device_offset)
{
  // the reference's device rule: rank % ndev + offset (deviceManager_OpenACC.cpp:31-50)
  b200_overlay::check(b200_init(rank, device_offset), "init_alt_B200");
  bool ok = true;
  ok &= AFopr<AFIELD_d>::init_factory();
  ok &= AFopr<AFIELD_f>::init_factory();
  ok &= ASolver<AFIELD_d>::init_factory();
  ok &= ASolver<AFIELD_f>::init_factory();
  return ok;
}
