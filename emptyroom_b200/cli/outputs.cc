// outputs.cc -- the .out report files, line for line in the reference's format
// (the format is the interface downstream scripts read).
#include "outputs.h"

#include <math.h>
#include <stdlib.h>
#include <time.h>

#include <vector>

void die(const std::string& message) {
    printf("%s\n", message.c_str());
    exit(EXIT_FAILURE);
}

void write_report_header(FILE* fh, const RunInfo& r, const er_structure* s,
                         const er_forcefield* f, const er_particle* parts) {
    time_t t = time(0);
    struct tm* now = localtime(&t);
    fprintf(fh, "date: %d-%d-%d\n\n", now->tm_year + 1900, now->tm_mon + 1, now->tm_mday);
    fprintf(fh, "Adsorbate: %s\n", r.adsorbate.c_str());
    fprintf(fh, "    Molecular weight = %f\n\n", r.adsorbate_mw);
    int n = 0;
    double cell[6], tm[9], vol, dens;
    er_structure_info(s, &n, cell, tm, nullptr, &vol, &dens);
    fprintf(fh, "Structure: %s\n", r.framework.c_str());
    fprintf(fh, "    Crystal density (kg/m3): %f\n", dens);
    fprintf(fh, "    a = %f A; b = %f A; c = %f A\n    alpha = %f, beta = %f, gamma = %f\n",
            cell[0], cell[1], cell[2], cell[3] / M_PI * 180.0, cell[4] / M_PI * 180.0,
            cell[5] / M_PI * 180.0);
    fprintf(fh, "    Atoms in framework: %d\n", n);
    fprintf(fh, "    Atom    # in framework\n");
    std::vector<std::string> labels(n);
    char buf[256];
    for (int i = 0; i < n; ++i) {
        er_structure_label(s, i, buf, sizeof(buf));
        labels[i] = buf;
    }
    const int nff = er_forcefield_count(f);
    for (int a = 0; a < nff; ++a) {
        er_forcefield_entry(f, a, buf, sizeof(buf), nullptr, nullptr);
        int count = 0;
        for (int k = 0; k < n; ++k)
            if (labels[k] == buf) ++count;
        if (count != 0) fprintf(fh, "    %s    %d\n", buf, count);
    }
    fprintf(fh, "\n    Tranformation matrix:\n");
    for (int i = 0; i < 3; ++i) {
        fprintf(fh, "    ");
        for (int j = 0; j < 3; ++j) fprintf(fh, " %f ", tm[3 * i + j]);
        fprintf(fh, "\n");
    }
    fprintf(fh, "\nForcefield: %s\n", r.forcefield.c_str());
    fprintf(fh, "    %s epsilon (K) = %f, sigma (A) = %f\n", r.adsorbate.c_str(), r.eps_guest,
            r.sig_guest);
    fprintf(fh, "    For LJ cutoff %f A, unit cell replication factors: %d %d %d\n",
            sqrt(r.r_cutoff_squared), r.rep[0], r.rep[1], r.rep[2]);
    fprintf(fh, "    %s-XX interactions present:\n    XX    epsilon(K)    sigma(A)\n",
            r.adsorbate.c_str());
    std::vector<std::string> printed;
    for (int i = 0; i < n; ++i) {
        bool seen = false;
        for (const std::string& p : printed)
            if (p == labels[i]) {
                seen = true;
                break;
            }
        if (seen) continue;
        printed.push_back(labels[i]);
        fprintf(fh, "    %s    %f    %f\n", labels[i].c_str(), parts[i].eps_with_adsorbate,
                sqrt(parts[i].sig_with_adsorbate_squared));
    }
}

void write_report_grid(FILE* fh, const RunInfo& r, const er_structure* s) {
    double cell[6];
    er_structure_info(s, nullptr, cell, nullptr, nullptr, nullptr, nullptr);
    fprintf(fh, "\nGrid: %d by %d by %d points. Total grid points = %d\n", r.nx, r.ny, r.nz,
            r.nx * r.ny * r.nz);
    fprintf(fh, "    Actual grid spacing: da = %f A, db = %f A, dc = %f A\n",
            cell[0] / (r.nx - 1), cell[1] / (r.ny - 1), cell[2] / (r.nz - 1));
}

void write_report_henry(FILE* fh, const RunInfo& r, const er_structure* s) {
    double vol = 0.0;
    er_structure_info(s, nullptr, nullptr, nullptr, nullptr, &vol, nullptr);
    fprintf(fh,
            "\nHenry info\n    # of blocks: %d\n    # of threads: %d\n    # of insertions per "
            "thread: %d\n",
            r.num_blocks, r.num_threads, r.per_thread);
    fprintf(fh, "    Specified # of insertions/ A3: %d\n", r.per_a3);
    fprintf(fh, "    Actual # of insertions/ A3: %f\n",
            r.per_thread * r.num_blocks * r.num_threads / vol);
    fprintf(fh, "    Total # of insertions: %d\n", r.per_thread * r.num_blocks * r.num_threads);
}
