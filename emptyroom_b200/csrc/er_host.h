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
    std::vector<double> img_lj64;       // 2 per image: its atom's C12, C6 in FP64
};

// Validates desc and fills everything of `out` but the image cell list
// (img_*, cell_start, nc, cell_lo stay empty): the scalars, and per atom the
// FP64 fractional position and sig2 (atom_frac), the FP64 (C12, C6)
// (atom_lj64) and the FP32 image coefficients (C12, -C6) in atom_par, which
// is (0, 0) for an atom with eps == 0 or sig2 == 0 (it has no images). The
// three per-atom arrays are written to the caller's buffers of n_atoms
// entries. w gets the perpendicular widths, *keep the image-keep distance.
int prepare_framework(const er_framework_desc& desc, double h, HostFramework& out,
                      std::string& err, HostImage* atom_frac, double* atom_lj64,
                      float* atom_par, double w[3], double* keep);

// Cell grid of edge h over the bounding box [lo, hi] of the kept images:
// sets f.cell_lo and f.nc; ER_ERR_LIMIT past 64 Mi cells.
int cell_grid(const double lo[3], const double hi[3], double h, HostFramework& f, int64_t* ncell,
              std::string& err);

// Validates desc and builds the image cell list with cell edge h (A).
int build_framework(const er_framework_desc& desc, double h, HostFramework& out,
                    std::string& err);

// Upper-triangular frame r = Q^T t of the cell matrix t (Q a proper rotation):
// r == t bit for bit when t[3] == t[6] == 0.
void positioning_frame(const double t[9], double r[9]);

// Perpendicular widths of the cell spanned by the columns of t (A).
void perpendicular_widths(const double t[9], double w[3]);

}  // namespace er
