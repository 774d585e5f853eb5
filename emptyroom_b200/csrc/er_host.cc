// er_host.cc -- host-side framework preparation and the C-ABI host helpers.
#include "er_host.h"

#include <math.h>
#include <string.h>

#include <algorithm>
#include <cstdio>

#include "er_philox.h"

namespace er {

static void cross(const double a[3], const double b[3], double c[3]) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

void positioning_frame(const double t[9], double r[9]) {
    if (t[3] == 0.0 && t[6] == 0.0) {
        for (int k = 0; k < 9; ++k) r[k] = t[k];
        return;
    }
    // Gram-Schmidt on the columns a, b, c: q1 = a/|a|, q2 = b' / |b'|,
    // q3 = q1 x q2 (a proper rotation, so handedness is kept)
    const double a[3] = {t[0], t[3], t[6]}, b[3] = {t[1], t[4], t[7]}, c[3] = {t[2], t[5], t[8]};
    const double la = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    const double q1[3] = {a[0] / la, a[1] / la, a[2] / la};
    const double r01 = q1[0] * b[0] + q1[1] * b[1] + q1[2] * b[2];
    double bp[3] = {b[0] - r01 * q1[0], b[1] - r01 * q1[1], b[2] - r01 * q1[2]};
    const double r11 = sqrt(bp[0] * bp[0] + bp[1] * bp[1] + bp[2] * bp[2]);
    const double q2[3] = {bp[0] / r11, bp[1] / r11, bp[2] / r11};
    double q3[3];
    cross(q1, q2, q3);
    r[0] = la;  r[1] = r01; r[2] = q1[0] * c[0] + q1[1] * c[1] + q1[2] * c[2];
    r[3] = 0.0; r[4] = r11; r[5] = q2[0] * c[0] + q2[1] * c[1] + q2[2] * c[2];
    r[6] = 0.0; r[7] = 0.0; r[8] = q3[0] * c[0] + q3[1] * c[1] + q3[2] * c[2];
}

void perpendicular_widths(const double t[9], double w[3]) {
    // columns of t are the cell vectors a, b, c
    const double a[3] = {t[0], t[3], t[6]}, b[3] = {t[1], t[4], t[7]}, c[3] = {t[2], t[5], t[8]};
    double bc[3], ca[3], ab[3];
    cross(b, c, bc);
    cross(c, a, ca);
    cross(a, b, ab);
    const double vol = fabs(a[0] * bc[0] + a[1] * bc[1] + a[2] * bc[2]);
    w[0] = vol / sqrt(bc[0] * bc[0] + bc[1] * bc[1] + bc[2] * bc[2]);
    w[1] = vol / sqrt(ca[0] * ca[0] + ca[1] * ca[1] + ca[2] * ca[2]);
    w[2] = vol / sqrt(ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2]);
}

int prepare_framework(const er_framework_desc& d, double h, HostFramework& f, std::string& err,
                      HostImage* atom_frac, double* atom_lj64, float* atom_par, double w[3],
                      double* keep) {
    if (d.n_atoms < 0 || (d.n_atoms > 0 && d.atoms == nullptr)) {
        err = "framework: n_atoms < 0 or atoms == NULL";
        return ER_ERR_INVALID;
    }
    for (int k = 0; k < 3; ++k) {
        if (d.rep[k] < 0 || d.rep[k] > 64) {
            err = "framework: replication factors must be in [0, 64]";
            return ER_ERR_INVALID;
        }
    }
    for (int k = 0; k < 9; ++k) {
        if (!std::isfinite(d.t_matrix[k])) {
            err = "framework: t_matrix has a non-finite entry";
            return ER_ERR_INVALID;
        }
    }
    if (!(d.r_cutoff_squared > 0.0) || !std::isfinite(d.r_cutoff_squared)) {
        err = "framework: r_cutoff_squared must be positive and finite";
        return ER_ERR_INVALID;
    }
    perpendicular_widths(d.t_matrix, w);
    if (!(w[0] > 0) || !(w[1] > 0) || !(w[2] > 0)) {
        err = "framework: degenerate cell matrix";
        return ER_ERR_INVALID;
    }
    const int64_t ipa = (int64_t)(2 * d.rep[0] + 1) * (2 * d.rep[1] + 1) * (2 * d.rep[2] + 1);
    if ((int64_t)d.n_atoms * ipa >= (int64_t)UINT32_MAX) {
        err = "framework: n_atoms * images exceeds the 32-bit image id range";
        return ER_ERR_LIMIT;
    }
    f = HostFramework();
    f.n_atoms = d.n_atoms;
    for (int k = 0; k < 3; ++k) f.rep[k] = d.rep[k];
    for (int k = 0; k < 9; ++k) f.t[k] = d.t_matrix[k];
    positioning_frame(d.t_matrix, f.r);
    f.rc2 = d.r_cutoff_squared;
    f.imgs_per_atom = (int)ipa;
    f.h = h;
    for (int a = 0; a < d.n_atoms; ++a) {
        const er_particle& p = d.atoms[a];
        if (!std::isfinite(p.x_f) || !std::isfinite(p.y_f) || !std::isfinite(p.z_f) ||
            !std::isfinite(p.eps_with_adsorbate) || !std::isfinite(p.sig_with_adsorbate_squared) ||
            p.eps_with_adsorbate < 0.0 || p.sig_with_adsorbate_squared < 0.0) {
            err = "framework: atom with non-finite or negative parameters";
            return ER_ERR_INVALID;
        }
        atom_frac[a] = HostImage{p.x_f, p.y_f, p.z_f, p.sig_with_adsorbate_squared};
        const double s2 = p.sig_with_adsorbate_squared;
        const double c6l = 4.0 * p.eps_with_adsorbate * s2 * s2 * s2;
        atom_lj64[2 * a] = c6l * s2 * s2 * s2;
        atom_lj64[2 * a + 1] = c6l;
    }
    for (int a = 0; a < d.n_atoms; ++a) {
        const er_particle& p = d.atoms[a];
        const double s2 = p.sig_with_adsorbate_squared;
        // An atom with eps == 0 or sig == 0 adds exactly 0.0 to every sum of
        // src/computegridsheet.h:82 (r^2 >= min_r^2 keeps s^6 finite): it
        // gets no images.
        atom_par[2 * a] = 0.0f;
        atom_par[2 * a + 1] = 0.0f;
        if (p.eps_with_adsorbate == 0.0 || s2 == 0.0) continue;
        const double s6 = s2 * s2 * s2;
        const double c6 = 4.0 * p.eps_with_adsorbate * s6;
        const double c12 = c6 * s6;
        float c12f = (float)c12;
        float c6f = (float)c6;
        if (!std::isfinite(c12f) || !std::isfinite(c6f)) {
            err = "framework: mixed LJ coefficients overflow FP32";
            return ER_ERR_LIMIT;
        }
        if (c12f == 0.0f) c12f = 1.17549435e-38f;  // keep u3 * (C12 u3 - C6) NaN-free
        atom_par[2 * a] = c12f;
        atom_par[2 * a + 1] = -c6f;
    }
    // Keep image a + n only if it can be within rc of the grid region
    // [0,1]^3: its fractional overshoot of slab d times the slab width w_d is a
    // lower bound on its distance to every grid point.
    const double rc = sqrt(d.r_cutoff_squared);
    *keep = rc * (1.0 + 1e-9) + 1e-6;
    return ER_OK;
}

int build_framework(const er_framework_desc& d, double h, HostFramework& f, std::string& err) {
    const int na = d.n_atoms > 0 ? d.n_atoms : 0;
    std::vector<HostImage> af(na);
    std::vector<double> lj(2 * (size_t)na);
    std::vector<float> apar(2 * (size_t)na);
    double w[3], keep = 0.0;
    const int st = prepare_framework(d, h, f, err, af.data(), lj.data(), apar.data(), w, &keep);
    if (st != ER_OK) return st;
    f.atom_frac = std::move(af);
    f.atom_lj64 = std::move(lj);
    const int64_t ipa = f.imgs_per_atom;
    std::vector<HostImage> xyz;
    std::vector<float> par;
    std::vector<uint32_t> ids;
    const double* t = f.r;  // image positions in the positioning frame
    for (int a = 0; a < d.n_atoms; ++a) {
        const er_particle& p = d.atoms[a];
        if (apar[2 * a] == 0.0f) continue;  // no images (eps == 0 or sig == 0)
        const float c12f = apar[2 * a], nc6f = apar[2 * a + 1];
        int code = 0;
        for (int i = -d.rep[0]; i <= d.rep[0]; ++i)
            for (int j = -d.rep[1]; j <= d.rep[1]; ++j)
                for (int k = -d.rep[2]; k <= d.rep[2]; ++k, ++code) {
                    const double fx = p.x_f + i, fy = p.y_f + j, fz = p.z_f + k;
                    const double ox = fx < 0 ? -fx : (fx > 1 ? fx - 1 : 0);
                    const double oy = fy < 0 ? -fy : (fy > 1 ? fy - 1 : 0);
                    const double oz = fz < 0 ? -fz : (fz > 1 ? fz - 1 : 0);
                    if (ox * w[0] >= keep || oy * w[1] >= keep || oz * w[2] >= keep) continue;
                    HostImage im;
                    im.x = t[0] * fx + t[1] * fy + t[2] * fz;
                    im.y = t[3] * fx + t[4] * fy + t[5] * fz;
                    im.z = t[6] * fx + t[7] * fy + t[8] * fz;
                    im.pad = 0.0;
                    xyz.push_back(im);
                    par.push_back(c12f);
                    par.push_back(nc6f);
                    ids.push_back((uint32_t)((int64_t)a * ipa + code));
                }
    }
    const size_t n = xyz.size();
    if (n >= (size_t)INT32_MAX) {
        err = "framework: too many images";
        return ER_ERR_LIMIT;
    }
    // cell list over the bounding box of the kept images
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    if (n > 0) {
        lo[0] = hi[0] = xyz[0].x;
        lo[1] = hi[1] = xyz[0].y;
        lo[2] = hi[2] = xyz[0].z;
        for (const HostImage& im : xyz) {
            lo[0] = std::min(lo[0], im.x); hi[0] = std::max(hi[0], im.x);
            lo[1] = std::min(lo[1], im.y); hi[1] = std::max(hi[1], im.y);
            lo[2] = std::min(lo[2], im.z); hi[2] = std::max(hi[2], im.z);
        }
    }
    int64_t ncell = 0;
    if (int st2 = cell_grid(lo, hi, h, f, &ncell, err)) return st2;
    std::vector<int> cell(n);
    std::vector<int> count((size_t)ncell + 1, 0);
    const double inv_h = 1.0 / h;
    for (size_t q = 0; q < n; ++q) {
        int c[3];
        const double v[3] = {xyz[q].x, xyz[q].y, xyz[q].z};
        for (int k = 0; k < 3; ++k) {
            c[k] = (int)floor((v[k] - f.cell_lo[k]) * inv_h);
            c[k] = std::min(std::max(c[k], 0), f.nc[k] - 1);
        }
        cell[q] = (c[2] * f.nc[1] + c[1]) * f.nc[0] + c[0];
        count[(size_t)cell[q] + 1]++;
    }
    for (int64_t c = 0; c < ncell; ++c) count[c + 1] += count[c];
    f.cell_start = count;
    f.img_xyz.resize(n);
    f.img_par.resize(2 * n);
    f.img_id.resize(n);
    f.img_lj64.resize(2 * n);
    std::vector<int> fill(count.begin(), count.end() - 1);
    for (size_t q = 0; q < n; ++q) {
        const int dst = fill[cell[q]]++;
        f.img_xyz[dst] = xyz[q];
        f.img_par[2 * dst] = par[2 * q];
        f.img_par[2 * dst + 1] = par[2 * q + 1];
        f.img_id[dst] = ids[q];
        const size_t a = ids[q] / (uint32_t)ipa;
        f.img_lj64[2 * dst] = f.atom_lj64[2 * a];
        f.img_lj64[2 * dst + 1] = f.atom_lj64[2 * a + 1];
    }
    return ER_OK;
}

int cell_grid(const double lo[3], const double hi[3], double h, HostFramework& f, int64_t* ncell,
              std::string& err) {
    int64_t nc = 1;
    for (int k = 0; k < 3; ++k) {
        f.cell_lo[k] = lo[k];
        f.nc[k] = (int)floor((hi[k] - lo[k]) / h) + 1;
        nc *= f.nc[k];
    }
    if (nc > (int64_t)64 * 1024 * 1024) {
        err = "framework: cell list too large (cell edge too small for this cell)";
        return ER_ERR_LIMIT;
    }
    *ncell = nc;
    return ER_OK;
}

}  // namespace er

// ------------------------------------------------------------------ C ABI helpers
extern "C" {

const char* er_status_string(int s) {
    switch (s) {
        case ER_OK: return "ok";
        case ER_ERR_INVALID: return "invalid argument";
        case ER_ERR_CUDA: return "CUDA error";
        case ER_ERR_NOMEM: return "out of memory";
        case ER_ERR_IO: return "I/O error";
        case ER_ERR_NOT_FOUND: return "not found";
        case ER_ERR_TIMEOUT: return "timed out";
        case ER_ERR_LIMIT: return "size limit exceeded";
        default: return "unknown status";
    }
}

const char* er_version(void) { return "emptyroom_b200 0.1 (sm_100a)"; }

int er_cell_matrices(double a, double b, double c, double alpha_deg, double beta_deg,
                     double gamma_deg, double t[9], double inv[9], double* volume) {
    // src/Framework.cc:35-37 (degrees -> radians) and :113-142
    const double al = alpha_deg * M_PI / 180.0;
    const double be = beta_deg * M_PI / 180.0;
    const double ga = gamma_deg * M_PI / 180.0;
    const double arg = 1.0 - pow(cos(al), 2.0) - pow(cos(be), 2) - pow(cos(ga), 2) +
                       2 * cos(al) * cos(be) * cos(ga);
    if (!(a > 0) || !(b > 0) || !(c > 0) || !(arg > 0) || sin(ga) == 0.0) return ER_ERR_INVALID;
    const double v = sqrt(arg);
    if (volume) *volume = v * a * b * c;
    if (t) {
        t[0] = a; t[1] = b * cos(ga); t[2] = c * cos(be);
        t[3] = 0.0; t[4] = b * sin(ga); t[5] = c * (cos(al) - cos(be) * cos(ga)) / sin(ga);
        t[6] = 0.0; t[7] = 0.0; t[8] = c * v / sin(ga);
    }
    if (inv) {
        inv[0] = 1.0 / a;
        inv[1] = -cos(ga) / a / sin(ga);
        inv[2] = (cos(al) * cos(ga) - cos(be)) / (a * v * sin(ga));
        inv[3] = 0.0;
        inv[4] = 1.0 / b / sin(ga);
        inv[5] = (cos(be) * cos(ga) - cos(al)) / (b * v * sin(ga));
        inv[6] = 0.0;
        inv[7] = 0.0;
        inv[8] = sin(ga) / (c * v);
    }
    return ER_OK;
}

int er_replication_factors(const double t[9], double r_cutoff, int factor, int rep[3]) {
    if (!t || !rep || !(r_cutoff > 0) || factor < 1) return ER_ERR_INVALID;
    double w[3];
    er::perpendicular_widths(t, w);
    for (int k = 0; k < 3; ++k) {
        if (!(w[k] > 0)) return ER_ERR_INVALID;
        rep[k] = (int)floor(factor * r_cutoff / w[k]) + 1;
    }
    return ER_OK;
}

void er_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    er::philox4x32_10(ctr, key, out);
}

void er_insertion_point(uint64_t seed, uint64_t i, double out[3]) {
    er::insertion_point(seed, i, out);
}

int er_synth_positions(uint64_t seed, const double t[9], int n_atoms, double d_min,
                       double* frac) {
    if (!t || (n_atoms > 0 && !frac) || n_atoms < 0 || d_min < 0) return ER_ERR_INVALID;
    // Random sequential addition: candidates from the Philox stream (counter
    // = attempt index, key = seed, lane 2 = 7), accepted when no accepted atom
    // lies within d_min under the 27 nearest periodic images.
    double w[3];
    er::perpendicular_widths(t, w);
    const double dm2 = d_min * d_min;
    int nb[3];
    for (int k = 0; k < 3; ++k) {
        nb[k] = d_min > 0 ? std::max(1, (int)floor(w[k] / std::max(d_min, 1e-3))) : 1;
        nb[k] = std::min(nb[k], 256);
    }
    // Bins in fractional space; a bin is at least d_min wide in Cartesian.
    std::vector<std::vector<int>> bins((size_t)nb[0] * nb[1] * nb[2]);
    const int64_t max_attempts = (int64_t)n_atoms * 2000 + 100000;
    int n = 0;
    for (int64_t att = 0; n < n_atoms && att < max_attempts; ++att) {
        const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
        const uint32_t ctr[4] = {(uint32_t)att, (uint32_t)((uint64_t)att >> 32), 7u, 0u};
        uint32_t r[4], r2[4];
        er::philox4x32_10(ctr, key, r);
        const uint32_t ctr2[4] = {(uint32_t)att, (uint32_t)((uint64_t)att >> 32), 8u, 0u};
        er::philox4x32_10(ctr2, key, r2);
        const double f[3] = {er::u53(r[0], r[1]), er::u53(r[2], r[3]), er::u53(r2[0], r2[1])};
        int b[3];
        for (int k = 0; k < 3; ++k) b[k] = std::min(nb[k] - 1, (int)(f[k] * nb[k]));
        bool ok = true;
        if (d_min > 0) {
            for (int di = -1; di <= 1 && ok; ++di)
                for (int dj = -1; dj <= 1 && ok; ++dj)
                    for (int dk = -1; dk <= 1 && ok; ++dk) {
                        const int bi = (b[0] + di + nb[0]) % nb[0];
                        const int bj = (b[1] + dj + nb[1]) % nb[1];
                        const int bk = (b[2] + dk + nb[2]) % nb[2];
                        for (int q : bins[((size_t)bi * nb[1] + bj) * nb[2] + bk]) {
                            double d0 = f[0] - frac[3 * q], d1 = f[1] - frac[3 * q + 1],
                                   d2 = f[2] - frac[3 * q + 2];
                            d0 -= floor(d0 + 0.5);
                            d1 -= floor(d1 + 0.5);
                            d2 -= floor(d2 + 0.5);
                            // nearest images around the wrapped difference
                            for (int ii = -1; ii <= 1 && ok; ++ii)
                                for (int jj = -1; jj <= 1 && ok; ++jj)
                                    for (int kk = -1; kk <= 1 && ok; ++kk) {
                                        const double e0 = d0 + ii, e1 = d1 + jj, e2 = d2 + kk;
                                        const double x = t[0] * e0 + t[1] * e1 + t[2] * e2;
                                        const double y = t[3] * e0 + t[4] * e1 + t[5] * e2;
                                        const double z = t[6] * e0 + t[7] * e1 + t[8] * e2;
                                        if (x * x + y * y + z * z < dm2) ok = false;
                                    }
                            if (!ok) break;
                        }
                    }
        }
        if (!ok) continue;
        frac[3 * n] = f[0];
        frac[3 * n + 1] = f[1];
        frac[3 * n + 2] = f[2];
        bins[((size_t)b[0] * nb[1] + b[1]) * nb[2] + b[2]].push_back(n);
        ++n;
    }
    return n == n_atoms ? ER_OK : ER_ERR_LIMIT;
}

}  // extern "C"
