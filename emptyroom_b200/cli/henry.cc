// henry -- drop-in for the reference's `henry <structure> <adsorbate>`
// (src/henry.cu:43-175): same inputs and output_files/<fw>_<ads>_henry.out.
// The insertion count keeps the reference's decomposition (64 x 256 x
// (N / 16384 + 1)) so the statistics are comparable; the insertion points
// come from the Philox4x32-10 stream with seed 1234 instead of MTGP32.
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
        printf("Run as:\n./henry structure_name AdsorbateID\n");
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
    if (er_read_settings("simulation.input", ER_SETTINGS_HENRY, &set, err, sizeof(err)) != ER_OK)
        die(err);
    r.forcefield = set.forcefield;
    r.r_cutoff_squared = set.r_cutoff_squared;
    if (er_read_uc(root, r.framework.c_str(), "once", r.rep, err, sizeof(err)) != ER_OK) die(err);
    er_forcefield* ff = nullptr;
    if (er_forcefield_load(root, r.forcefield.c_str(), &ff, err, sizeof(err)) != ER_OK) die(err);
    er_structure* st = nullptr;
    if (er_structure_load(root, r.framework.c_str(), &st, err, sizeof(err)) != ER_OK) die(err);
    int n = 0;
    double t[9], vol = 0, dens = 0;
    er_structure_info(st, &n, nullptr, t, nullptr, &vol, &dens);
    // src/henry.cu:79, :94-95
    const int numinsertions = (int)(set.insertions_per_a3 * vol);
    if (er_forcefield_find(ff, r.adsorbate.c_str(), &r.eps_guest, &r.sig_guest) != ER_OK)
        die("Could not find adsorbate " + r.adsorbate + " in forcefield file " + r.forcefield);
    std::vector<er_particle> parts(n);
    if (er_mix_particles(st, ff, r.eps_guest, r.sig_guest, parts.data(), err, sizeof(err)) !=
        ER_OK)
        die(err);
    r.num_blocks = 64;
    r.num_threads = 256;
    r.per_thread = numinsertions / (r.num_blocks * r.num_threads) + 1;
    r.per_a3 = set.insertions_per_a3;
    const std::string outname = "output_files/" + r.framework + "_" + r.adsorbate + "_henry.out";
    FILE* out = fopen(outname.c_str(), "w");
    if (!out) die("Could not open " + outname);
    write_report_header(out, r, st, ff, parts.data());
    write_report_henry(out, r, st);

    er_ctx* ctx = nullptr;
    if (er_ctx_create(0, &ctx) != ER_OK) die("No usable CUDA device for henry");
    er_framework_desc d;
    d.n_atoms = n;
    d.atoms = parts.data();
    for (int k = 0; k < 9; ++k) d.t_matrix[k] = t[k];
    for (int k = 0; k < 3; ++k) d.rep[k] = r.rep[k];
    d.r_cutoff_squared = r.r_cutoff_squared;
    int fw = 0;
    if (er_framework_upload(ctx, &d, &fw) != ER_OK) die(er_ctx_last_error(ctx));
    const int64_t total = (int64_t)r.per_thread * r.num_blocks * r.num_threads;
    const double t0 = wall();
    er_henry_result res;
    if (er_henry(ctx, fw, set.temperature, total, 1234, nullptr, 0, 0, 0, &res, nullptr) != ER_OK)
        die(er_ctx_last_error(ctx));
    const double sim_time = wall() - t0;
    // src/henry.cu:152-174
    fprintf(out, "\nHenry simulation results\n");
    fprintf(out, "    Simulation time: %f s\n", sim_time);
    const double ensemble_average_energy = res.sum_ew / res.sum_w;
    const double henry_coeff = res.sum_w / (double)total / set.temperature / 8.314;
    fprintf(out, "    Temperature (K): %f\n", set.temperature);
    fprintf(out, "    <energy> (kJ/mol): %f\n", ensemble_average_energy * 8.314 / 1000.0);
    fprintf(out, "    <energy> (K): %f\n", ensemble_average_energy);
    fprintf(out, "    Henry coefficient (mol/(kg-Pa)): %e\n", henry_coeff / dens);
    fprintf(out, "    Henry coefficient (mol/(m3-Pa)): %e\n", henry_coeff);
    fclose(out);
    er_ctx_destroy(ctx);
    er_structure_free(st);
    er_forcefield_free(ff);
    return 0;
}
