// Entry point of the B200 alt implementation for the reference driver:
// called where the Accel build calls init_alt_Accel (src/lib_alt_Accel/
// init_alt_Accel.cpp:20-49), it selects the GPU and registers
// "Domainwall_5din_eo" for AFopr<AField<double|float, B200>> and "CG" for
// ASolver<AField<double|float, B200>> in the reference's factories.
#ifndef B200_INIT_ALT_B200_INCLUDED
#define B200_INIT_ALT_B200_INCLUDED

bool init_alt_B200(int rank, int device_offset);

#endif
