/* Stand-in for the MSVC fopen_s the reference's case generator calls
 * (generateSimulationCases/genParticlesFunctions.cpp); test infrastructure. */
#ifndef ORACLE_FOPEN_S_H
#define ORACLE_FOPEN_S_H
#include <stdio.h>
static inline int fopen_s(FILE** f, const char* name, const char* mode)
{
    *f = fopen(name, mode);
    return *f ? 0 : 1;
}
#endif
