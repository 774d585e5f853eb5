// er_internal.h -- data layouts shared by the host side and the kernels.
#pragma once
#include <stdint.h>

#include <cuda_runtime.h>

namespace er {

// Device view of one uploaded framework/probe pair.
//
// Atom images a + T n (n in [-rep, rep]^3, the image loop of
// src/computegridsheet.h:54-56) that can lie within the cutoff of the unit
// cell are kept, sorted into a Cartesian cell list whose x index runs fastest,
// so one (y, z) row of cells is one contiguous range of images. Cartesian
// positions are taken in the frame r (the first lattice axis along x).
struct FwDev {
    const double4* img_xyz;   // Cartesian position (x, y, z, 0), FP64, cell-sorted
    const float2* img_par;    // (C12, -C6) = (4 eps sig^12, -4 eps sig^6), FP32
    const uint32_t* img_id;   // atom * imgs_per_atom + image code
    const int* cell_start;    // nc0*nc1*nc2 + 1 offsets into the image arrays
    const double4* atom_frac; // FP64 fractional (x_f, y_f, z_f, sig2) per atom
    const double2* atom_lj64; // FP64 (C12, C6) per atom
    const double2* img_lj64;  // FP64 (C12, C6) per image (near pairs of PREC_NEAR64)
    int n_img;
    int n_atoms;
    int nc[3];                // cells per axis
    double cell_lo[3];        // Cartesian corner of cell (0,0,0)
    double h, inv_h;          // cell edge (A)
    double t[9];              // fractional -> Cartesian (the caller's cell matrix), row-major
    double r[9];              // positioning frame: upper-triangular rotation of t (== t
                              // when t is upper triangular); positions use r
    double rc2;               // squared cutoff, FP64 (the reference's r_cutoff_squared)
    int rep[3];
    int imgs_per_atom;        // (2 rep0 + 1)(2 rep1 + 1)(2 rep2 + 1)
    int* fault;               // set to 1 by a kernel whose bounded wait gave up (the
                              // context's mapped fault word; may be null)
};

// Per-launch constants derived from the cutoff.
struct CutoffConsts {
    float rc2f;      // fl32(rc2)
    float rin2;      // (rc - margin)^2: inside for every point of a warp box
    float rout2;     // (rc + margin)^2: possibly inside
    double rc;       // cutoff radius (A)
    double rcm;      // rc + margin (CTA candidate radius)
    double r2min;    // clamp of the reference (min_r^2)
};

// One grid job (a framework and an nx x ny x nz lattice, axes i/(N-1)).
struct GridTask {
    FwDev fw;
    CutoffConsts cc;
    int nx, ny, nz;
    int nb[3];          // bricks per axis
    int tile_p;         // points per thread of the kernel variant (brick 2P x 8 x 16)
    float* out;         // nx*ny*nz, index k + j*nz + i*ny*nz
    double* out64;      // same layout, FP64 (PREC_FP64 jobs only)
};

// Widom points of one framework. `order` lists the unblocked insertion indices
// sorted by spatial bin (bins in 2x2x2 brick order, ascending index inside a
// bin), so 128 consecutive entries (one warp) form a compact cluster.
struct PointTask {
    FwDev fw;
    CutoffConsts cc;
    const double* pts;       // FP64 Cartesian points (frame r), 3 per entry of `order`
                             // (bin order)
    const int* order;        // unblocked insertion indices in bin order
    uint64_t seed;           // Philox stream of the points (fractional coordinates are
                             // regenerated from it for the exact cutoff decisions)
    const int* n_valid;      // device count of entries in `order`
    float* energies;         // E per insertion (insertion order)
};

// Persistent-queue item as the kernel decodes it: (task position, brick).
struct WorkItem {
    int task;
    int brick;
};

}  // namespace er
