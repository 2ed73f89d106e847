// main_loop.cpp -- the reference's time loop (VoxarMPS/VoxarMPS/main.cu:
// 1027-1363) driven through include/voxarmps.h from C++, the way
// INTEGRATION.md shows it.  Built and run by tests/test_gpu_cpp.py.
//
//   main_loop <config.bin> <input.grd> <steps> <step|stages> <out.bin>
//
// config.bin holds one mps_config (the caller fills it from its constants);
// the particles come from a .grd file (main.cu:496-684).  "step" calls
// mps_step once per iteration, "stages" calls the fourteen per-stage entry
// points in main.cu's order.  The state is read back into 1-based host
// arrays, as the reference keeps them, and written to out.bin as
// TP, then x y z u v w p (TP doubles each, caller order).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "voxarmps.h"

static int fail(const char* what, int st, mps_ctx* ctx)
{
    fprintf(stderr, "%s: status %d (%s)\n", what, st, ctx ? mps_last_message(ctx) : "");
    return 1;
}

#define CALL(x)                                     \
    do {                                            \
        int _st = (x);                              \
        if (_st != MPS_OK) return fail(#x, _st, ctx); \
    } while (0)

int main(int argc, char** argv)
{
    if (argc != 6) {
        fprintf(stderr, "usage: %s config.bin input.grd steps step|stages out.bin\n", argv[0]);
        return 2;
    }
    mps_config cfg;
    FILE* f = fopen(argv[1], "rb");
    if (!f || fread(&cfg, sizeof(cfg), 1, f) != 1) {
        fprintf(stderr, "cannot read %s\n", argv[1]);
        return 2;
    }
    fclose(f);
    const int steps = atoi(argv[3]);
    const bool staged = strcmp(argv[4], "stages") == 0;
    mps_ctx* ctx = nullptr;
    CALL(mps_create(&cfg, 0, &ctx));
    CALL(mps_load_grd(ctx, argv[2]));
    CALL(mps_init(ctx));
    for (int t = 1; t <= steps; t++) {
        if (!staged) {
            CALL(mps_step(ctx));
            continue;
        }
        int iters = 0;
        double relres = 0;
        if (cfg.method != 3) CALL(mps_pnd(ctx));          // PNUM
        CALL(mps_neighbors(ctx));                          // NEIGHBOR
        if (cfg.turb) CALL(mps_sps(ctx));                  // SPS
        CALL(mps_vfraction(ctx));                          // V_FRACTION
        CALL(mps_viscosity(ctx));                          // VISCOSITY
        CALL(mps_predict(ctx));                            // PREDICTION
        CALL(mps_pnd_star(ctx));                           // PNUMSTAR
        if (cfg.method != 3) CALL(mps_bcon(ctx));          // BCON
        CALL(mps_pressure(ctx, &iters, &relres));          // PRESSURECALC
        CALL(mps_phat(ctx));                               // PHATCALC
        CALL(mps_pressure_gradient(ctx));                  // PRESSGRAD
        CALL(mps_integrate(ctx));                          // EULERINTEGRATION
        CALL(mps_collision(ctx));                          // COLLISION2
        CALL(mps_commit(ctx));                             // PREPDATA
    }
    double n_d = 0;
    CALL(mps_get_scalar(ctx, "n", &n_d));
    const int TP = (int)n_d;
    // 1-based host arrays, as main.cu allocates them (main.cu:554-563)
    std::vector<std::vector<double>> a(7, std::vector<double>((size_t)TP + 1, 0.0));
    const bool three = cfg.dim == 3;
    CALL(mps_get_state(ctx, &a[0][1], &a[1][1], three ? &a[2][1] : nullptr, &a[3][1], &a[4][1],
                       three ? &a[5][1] : nullptr, &a[6][1]));
    FILE* o = fopen(argv[5], "wb");
    if (!o) return fail("fopen", MPS_ERR_IO, ctx);
    fwrite(&TP, sizeof(int), 1, o);
    for (auto& v : a) fwrite(&v[1], sizeof(double), (size_t)TP, o);
    fclose(o);
    CALL(mps_destroy(ctx));
    printf("%d particles, %d steps (%s)\n", TP, steps, staged ? "stages" : "step");
    return 0;
}
