// Command-line driver for the reference's case generator (test
// infrastructure): gen <case> <DL> <mult> <out.grd> calls the reference's own
// createParticles* function (generateSimulationCases/genParticlesFunctions.h)
// so that voxarmps_b200/gen.py can be compared with its output.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "genParticlesFunctions.h"

int main(int argc, char** argv)
{
    if (argc != 5) {
        std::fprintf(stderr, "usage: gen <case> <DL> <mult> <out.grd>\n");
        return 2;
    }
    const char* c = argv[1];
    const double dl = std::atof(argv[2]), mult = std::atof(argv[3]);
    const char* out = argv[4];
    if (!std::strcmp(c, "oil_spill_2d")) createParticlesOilSpill2D(dl, mult, out);
    else if (!std::strcmp(c, "dam_break_2d")) createParticlesDamBreak2D(dl, mult, out);
    else if (!std::strcmp(c, "shear_cavity_2d")) createParticlesShearCavity2D(dl, mult, out);
    else if (!std::strcmp(c, "water_drop_2d")) createParticlesWaterDrop2D(dl, mult, out);
    else if (!std::strcmp(c, "rt_instability_2d")) createParticlesRTinstability(dl, mult, out);
    else if (!std::strcmp(c, "poiseuille_2d")) createParticlesPoiseuilleFlow2D(dl, mult, out);
    else if (!std::strcmp(c, "dam_break_3d")) createParticlesDamBreak3D(dl, mult, out);
    else if (!std::strcmp(c, "dam_break_3d_offset")) createParticlesDamBreak3D_offset_nozero(dl, mult, out);
    else return 2;
    return 0;
}
