// writegrid -- drop-in for the reference's `writegrid <structure> <adsorbate>`
// (src/writegrid.cu:52-323): same inputs (simulation.input, data/...), same
// outputs (data/grids/<fw>_<ads>_<ff>.txt|.cube and output_files/<fw>_<ads>_grid.out),
// run from the project root. The whole grid is computed in one call of the
// sm_100a library (er_grid) instead of one kernel launch per x-sheet, and the
// text is formatted on all host cores.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <sys/time.h>

#include <string>
#include <vector>

#include "../../include/emptyroom_b200.h"
#include "outputs.h"

static double wall() {
    struct timeval tv;
    gettimeofday(&tv, nullptr);
    return tv.tv_sec + 1e-6 * tv.tv_usec;
}

int main(int argc, char* argv[]) {
    if (argc != 3) {
        printf("Run as:\n./writegrid structure_name AdsorbateID\n");
        exit(EXIT_FAILURE);
    }
    char err[1024] = {0};
    RunInfo r;
    r.framework = argv[1];
    r.adsorbate = argv[2];
    const char* root = ".";
    if (er_adsorbate_mw(root, r.adsorbate.c_str(), &r.adsorbate_mw, err, sizeof(err)) != ER_OK)
        die(err);
    er_settings set;
    if (er_read_settings("simulation.input", ER_SETTINGS_GRID, &set, err, sizeof(err)) != ER_OK)
        die(err);
    if (set.verbose) printf("Read simulation.input\n");
    r.forcefield = set.forcefield;
    r.r_cutoff_squared = set.r_cutoff_squared;
    if (er_read_uc(root, r.framework.c_str(), "once", r.rep, err, sizeof(err)) != ER_OK) die(err);
    er_forcefield* ff = nullptr;
    if (er_forcefield_load(root, r.forcefield.c_str(), &ff, err, sizeof(err)) != ER_OK) die(err);
    er_structure* st = nullptr;
    if (er_structure_load(root, r.framework.c_str(), &st, err, sizeof(err)) != ER_OK) die(err);
    if (er_forcefield_find(ff, r.adsorbate.c_str(), &r.eps_guest, &r.sig_guest) != ER_OK)
        die("Could not find adsorbate " + r.adsorbate + " in forcefield file " + r.forcefield);
    int n = 0;
    double cell[6], t[9];
    er_structure_info(st, &n, cell, t, nullptr, nullptr, nullptr);
    std::vector<er_particle> parts(n);
    if (er_mix_particles(st, ff, r.eps_guest, r.sig_guest, parts.data(), err, sizeof(err)) !=
        ER_OK)
        die(err);
    // grid size and axes, src/writegrid.cu:110-127
    r.nx = (int)ceil(cell[0] / set.grid_resolution);
    r.ny = (int)ceil(cell[1] / set.grid_resolution);
    r.nz = (int)ceil(cell[2] / set.grid_resolution);
    const std::string fmt = set.grid_output_format;
    if (fmt != "txt" && fmt != "cube") die("Grid output format must be txt or cube");
    const std::string outname = "output_files/" + r.framework + "_" + r.adsorbate + "_grid.out";
    FILE* out = fopen(outname.c_str(), "w");
    if (!out) die("Could not open " + outname);
    write_report_header(out, r, st, ff, parts.data());
    write_report_grid(out, r, st);
    const std::string gridname =
        "data/grids/" + r.framework + "_" + r.adsorbate + "_" + r.forcefield + "." + fmt;
    fprintf(out, "    Size of framework atoms array = %f MB\n",
            n * sizeof(er_particle) / (1024.0 * 1024.0));
    fprintf(out, "    Size of grid = %f MB\n",
            (double)r.nx * r.ny * r.nz * sizeof(float) / (1024.0 * 1024.0));
    fprintf(out, "    A block is 256 threads over 8 x 8 x 16 grid points.\n");

    er_ctx* ctx = nullptr;
    if (er_ctx_create(0, &ctx) != ER_OK) die("No usable CUDA device for writegrid");
    er_framework_desc d;
    d.n_atoms = n;
    d.atoms = parts.data();
    for (int k = 0; k < 9; ++k) d.t_matrix[k] = t[k];
    for (int k = 0; k < 3; ++k) d.rep[k] = r.rep[k];
    d.r_cutoff_squared = r.r_cutoff_squared;
    const double t0 = wall();
    int fw = 0;
    if (er_framework_upload(ctx, &d, &fw) != ER_OK) die(er_ctx_last_error(ctx));
    std::vector<float> grid((size_t)r.nx * r.ny * r.nz);
    if (er_grid(ctx, fw, r.nx, r.ny, r.nz, ER_OUT_HOST | ER_OUT_F32, grid.data()) != ER_OK)
        die(er_ctx_last_error(ctx));
    int wst = fmt == "txt" ? er_write_grid_txt(gridname.c_str(), grid.data(), r.nx, r.ny, r.nz, 0)
                           : er_write_grid_cube(gridname.c_str(), grid.data(), r.nx, r.ny, r.nz,
                                                t, 0);
    if (wst != ER_OK) die("Could not write " + gridname);
    const double sim_time = wall() - t0;
    fprintf(out, "    Time to write grid: %f s\n", sim_time);
    if (set.verbose) printf("Completed grid writing!\n");
    fclose(out);
    er_ctx_destroy(ctx);
    er_structure_free(st);
    er_forcefield_free(ff);
    return 0;
}
