/*
 * ref_gcmc.cc -- the reference's own GCMC grid lookup on the host, as the
 * parity checker of oracle_grid_interp and er_grid_interp.
 *
 * TEST INFRASTRUCTURE ONLY. src/gcmc.cc does not compile as shipped, so
 * oracle/Makefile extracts its WrapToInterval, GetEnergyGridIndex and
 * GuestFrameworkEnergy functions verbatim into the build output
 * oracle/_ref/gcmc_interp.inc (never committed) and compiles them here with
 * the reference's src/datatypes.h.
 */
#include <math.h>
#include <stdint.h>

#include "datatypes.h"
#include "gcmc_interp.inc"

extern "C" void ref_grid_interp(double* grid, int nx, int ny, int nz, const double* pts,
                                int64_t n, double* out) {
    GridInfo gi;
    gi.N_x = nx;
    gi.N_y = ny;
    gi.N_z = nz;
    // src/gcmc.cc:343-345
    gi.dx_f = 1.0 / (gi.N_x - 1);
    gi.dy_f = 1.0 / (gi.N_y - 1);
    gi.dz_f = 1.0 / (gi.N_z - 1);
    gi.numtotalpts = nx * ny * nz;
    for (int64_t q = 0; q < n; ++q)
        // the call sites, src/gcmc.cc:191-194
        out[q] = GuestFrameworkEnergy(WrapToInterval(pts[3 * q], 1.0),
                                      WrapToInterval(pts[3 * q + 1], 1.0),
                                      WrapToInterval(pts[3 * q + 2], 1.0), gi, grid);
}
