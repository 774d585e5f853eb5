// er_host.h -- host-side preparation of framework data for the kernels.
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/emptyroom_b200.h"

namespace er {

struct HostImage {
    double x, y, z, pad;
};

// Everything the device needs for one framework/probe pair, built on the host.
struct HostFramework {
    int n_atoms = 0;
    int rep[3] = {0, 0, 0};
    int imgs_per_atom = 1;
    double t[9] = {0};
    double r[9] = {0};                  // positioning frame (upper triangular)
    double rc2 = 0.0;
    double h = 2.0;
    int nc[3] = {1, 1, 1};
    double cell_lo[3] = {0, 0, 0};
    std::vector<HostImage> img_xyz;     // cell-sorted Cartesian images
    std::vector<float> img_par;         // 2 per image: C12, -C6
    std::vector<uint32_t> img_id;       // atom * imgs_per_atom + image code
    std::vector<int> cell_start;        // nc0*nc1*nc2 + 1
    std::vector<HostImage> atom_frac;   // x_f, y_f, z_f, sig2 per atom
    std::vector<double> atom_lj64;      // 2 per atom: C12, C6 in FP64
};

// Validates desc and builds the image cell list with cell edge h (A).
int build_framework(const er_framework_desc& desc, double h, HostFramework& out,
                    std::string& err);

// Upper-triangular frame r = Q^T t of the cell matrix t (Q a proper rotation):
// r == t bit for bit when t[3] == t[6] == 0.
void positioning_frame(const double t[9], double r[9]);

// Perpendicular widths of the cell spanned by the columns of t (A).
void perpendicular_widths(const double t[9], double w[3]);

}  // namespace er
