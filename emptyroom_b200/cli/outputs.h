// outputs.h -- the .out report files of the writegrid / henry tools.
#pragma once
#include <stdio.h>

#include <string>

#include "../../include/emptyroom_b200.h"

struct RunInfo {
    std::string framework, adsorbate, forcefield;
    double adsorbate_mw = 0.0;
    double eps_guest = 0.0, sig_guest = 0.0;
    double r_cutoff_squared = 0.0;
    int rep[3] = {0, 0, 0};
    int nx = 0, ny = 0, nz = 0;                                   // grid
    int num_blocks = 0, num_threads = 0, per_thread = 0, per_a3 = 0;  // henry
};

// Header of the report: date, adsorbate, structure, cell, atom counts,
// transformation matrix, guest parameters and the mixed pairs
// (the common part of src/write_settings_to_outputfile.h:11-101 / :103-189).
void write_report_header(FILE* fh, const RunInfo& r, const er_structure* s,
                         const er_forcefield* f, const er_particle* parts);
// Grid section, src/write_settings_to_outputfile.h:87-100.
void write_report_grid(FILE* fh, const RunInfo& r, const er_structure* s);
// Henry section, src/write_settings_to_outputfile.h:178-188.
void write_report_henry(FILE* fh, const RunInfo& r, const er_structure* s);

// Prints "message\n" and exits with EXIT_FAILURE (the tools' error path).
[[noreturn]] void die(const std::string& message);
