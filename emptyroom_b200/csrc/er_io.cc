// er_io.cc -- the reference's input/output file formats (host side).
//
// The loaders read the same files, tokens and defaults as Framework
// (src/Framework.cc), Forcefield (src/Forcefield.cc) and readsettings.h, but
// report errors as status codes. The grid writers produce byte-identical text
// to the reference's fprintf loops, with the formatting split over threads.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <fstream>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "../../include/emptyroom_b200.h"

struct er_structure {
    std::string name;
    double a = 0, b = 0, c = 0, alpha = 0, beta = 0, gamma = 0;  // radians
    int n = 0;
    std::vector<double> x, y, z, mass;
    std::vector<std::string> label;
    double volume = 0, density = 0;
    double t[9] = {0}, inv[9] = {0};
};

struct er_forcefield {
    std::string name;
    std::vector<std::string> label;
    std::vector<double> eps, sig;
};

namespace {

void put_err(char* err, size_t len, const std::string& m) {
    if (err && len) {
        snprintf(err, len, "%s", m.c_str());
    }
}

std::string join(const char* root, const std::string& rel) {
    std::string r = root ? root : "";
    if (r.empty()) return rel;
    if (r.back() != '/') r += '/';
    return r + rel;
}

}  // namespace

extern "C" {

int er_structure_load(const char* root, const char* name, er_structure** out, char* err,
                      size_t errlen) {
    if (!name || !out) return ER_ERR_INVALID;
    *out = nullptr;
    const std::string cssr_name = std::string(name) + ".cssr";
    std::ifstream cssr(join(root, "data/structures/" + cssr_name).c_str());
    if (cssr.fail()) {  // src/Framework.cc:18-21
        put_err(err, errlen, "CSSR file " + cssr_name + " failed to import!");
        return ER_ERR_IO;
    }
    er_structure* s = new er_structure();
    s->name = name;
    std::string line;
    std::istringstream input;
    getline(cssr, line);
    input.str(line);
    input >> s->a >> s->b >> s->c;
    getline(cssr, line);
    input.str(line);
    input.clear();
    input >> s->alpha >> s->beta >> s->gamma;
    s->alpha = s->alpha * M_PI / 180.0;
    s->beta = s->beta * M_PI / 180.0;
    s->gamma = s->gamma * M_PI / 180.0;
    getline(cssr, line);
    input.str(line);
    input.clear();
    input >> s->n;
    if (s->n < 0 || s->n > 50000000) {
        delete s;
        put_err(err, errlen, "CSSR file " + cssr_name + ": bad atom count");
        return ER_ERR_INVALID;
    }
    s->x.resize(s->n);
    s->y.resize(s->n);
    s->z.resize(s->n);
    s->label.resize(s->n);
    s->mass.resize(s->n);
    getline(cssr, line);  // title line
    for (int i = 0; i < s->n; ++i) {
        if (!getline(cssr, line)) {
            delete s;
            put_err(err, errlen, "CSSR file " + cssr_name + ": fewer atom lines than declared");
            return ER_ERR_IO;
        }
        input.str(line);
        input.clear();
        int junk;
        input >> junk >> s->label[i] >> s->x[i] >> s->y[i] >> s->z[i];
        s->x[i] = fmod(s->x[i], 1.0);  // src/Framework.cc:58-60
        s->y[i] = fmod(s->y[i], 1.0);
        s->z[i] = fmod(s->z[i], 1.0);
    }
    // masses, src/Framework.cc:66-108
    const std::string mpath = "data/masses.def";
    std::ifstream mf(join(root, mpath).c_str());
    if (mf.fail()) {
        delete s;
        put_err(err, errlen, "File " + mpath + " not present.");
        return ER_ERR_IO;
    }
    getline(mf, line);
    std::vector<std::string> ids;
    std::vector<double> masses;
    while (getline(mf, line)) {
        input.str(line);
        input.clear();
        std::string id;
        double m = 0.0;
        input >> id >> m;
        ids.push_back(id);
        masses.push_back(m);
    }
    for (int k = 0; k < s->n; ++k) {
        bool found = false;
        for (size_t a = 0; a < ids.size(); ++a) {
            if (s->label[k] == ids[a]) {
                found = true;
                s->mass[k] = masses[a];
                break;
            }
        }
        if (!found) {
            put_err(err, errlen, "Atom " + s->label[k] + " not present in " + mpath + ".");
            delete s;
            return ER_ERR_NOT_FOUND;
        }
    }
    double vol = 0.0;
    if (er_cell_matrices(s->a, s->b, s->c, s->alpha * 180.0 / M_PI, s->beta * 180.0 / M_PI,
                         s->gamma * 180.0 / M_PI, s->t, s->inv, &vol) != ER_OK) {
        delete s;
        put_err(err, errlen, "CSSR file " + cssr_name + ": degenerate cell");
        return ER_ERR_INVALID;
    }
    // volume and density exactly as src/Framework.cc:113-119 (from radians)
    const double v_unit_piped = sqrt(1.0 - pow(cos(s->alpha), 2.0) - pow(cos(s->beta), 2) -
                                     pow(cos(s->gamma), 2) +
                                     2 * cos(s->alpha) * cos(s->beta) * cos(s->gamma));
    s->volume = v_unit_piped * s->a * s->b * s->c;
    double mass_uc = 0.0;
    for (int k = 0; k < s->n; ++k) mass_uc += s->mass[k];
    s->density = mass_uc / s->volume * 1660.53892;
    // transformation matrices from radians (src/Framework.cc:124-142)
    const double al = s->alpha, be = s->beta, ga = s->gamma;
    s->t[0] = s->a; s->t[1] = s->b * cos(ga); s->t[2] = s->c * cos(be);
    s->t[3] = 0.0; s->t[4] = s->b * sin(ga);
    s->t[5] = s->c * (cos(al) - cos(be) * cos(ga)) / sin(ga);
    s->t[6] = 0.0; s->t[7] = 0.0; s->t[8] = s->c * v_unit_piped / sin(ga);
    s->inv[0] = 1.0 / s->a;
    s->inv[1] = -cos(ga) / s->a / sin(ga);
    s->inv[2] = (cos(al) * cos(ga) - cos(be)) / (s->a * v_unit_piped * sin(ga));
    s->inv[3] = 0.0;
    s->inv[4] = 1.0 / s->b / sin(ga);
    s->inv[5] = (cos(be) * cos(ga) - cos(al)) / (s->b * v_unit_piped * sin(ga));
    s->inv[6] = 0.0;
    s->inv[7] = 0.0;
    s->inv[8] = sin(ga) / (s->c * v_unit_piped);
    *out = s;
    return ER_OK;
}

void er_structure_free(er_structure* s) { delete s; }

int er_structure_info(const er_structure* s, int* n_atoms, double cell[6], double t[9],
                      double inv[9], double* volume, double* density) {
    if (!s) return ER_ERR_INVALID;
    if (n_atoms) *n_atoms = s->n;
    if (cell) {
        cell[0] = s->a; cell[1] = s->b; cell[2] = s->c;
        cell[3] = s->alpha; cell[4] = s->beta; cell[5] = s->gamma;
    }
    if (t) memcpy(t, s->t, sizeof(s->t));
    if (inv) memcpy(inv, s->inv, sizeof(s->inv));
    if (volume) *volume = s->volume;
    if (density) *density = s->density;
    return ER_OK;
}

int er_structure_frac(const er_structure* s, double* frac) {
    if (!s || (s->n && !frac)) return ER_ERR_INVALID;
    for (int i = 0; i < s->n; ++i) {
        frac[3 * i] = s->x[i];
        frac[3 * i + 1] = s->y[i];
        frac[3 * i + 2] = s->z[i];
    }
    return ER_OK;
}

int er_structure_label(const er_structure* s, int i, char* buf, size_t len) {
    if (!s || !buf || !len || i < 0 || i >= s->n) return ER_ERR_INVALID;
    snprintf(buf, len, "%s", s->label[i].c_str());
    return ER_OK;
}

int er_forcefield_load(const char* root, const char* name, er_forcefield** out, char* err,
                       size_t errlen) {
    if (!name || !out) return ER_ERR_INVALID;
    *out = nullptr;
    const std::string rel = std::string("data/forcefields/") + name + ".def";
    std::ifstream f(join(root, rel).c_str());
    if (f.fail()) {  // src/Forcefield.cc:19-22
        put_err(err, errlen, "Forcefield file " + rel + " did not load.");
        return ER_ERR_IO;
    }
    er_forcefield* ff = new er_forcefield();
    ff->name = name;
    std::string line;
    getline(f, line);  // header
    while (getline(f, line)) {
        std::istringstream ss(line);
        std::string id;
        double e = 0.0, s = 0.0;
        ss >> id >> e >> s;
        ff->label.push_back(id);
        ff->eps.push_back(e);
        ff->sig.push_back(s);
    }
    *out = ff;
    return ER_OK;
}

void er_forcefield_free(er_forcefield* f) { delete f; }

int er_forcefield_count(const er_forcefield* f) { return f ? (int)f->label.size() : -1; }

int er_forcefield_entry(const er_forcefield* f, int i, char* label, size_t len, double* eps,
                        double* sig) {
    if (!f || i < 0 || i >= (int)f->label.size()) return ER_ERR_INVALID;
    if (label && len) snprintf(label, len, "%s", f->label[i].c_str());
    if (eps) *eps = f->eps[i];
    if (sig) *sig = f->sig[i];
    return ER_OK;
}

int er_forcefield_find(const er_forcefield* f, const char* label, double* eps, double* sig) {
    if (!f || !label) return ER_ERR_INVALID;
    for (size_t i = 0; i < f->label.size(); ++i) {
        if (f->label[i] == label) {
            if (eps) *eps = f->eps[i];
            if (sig) *sig = f->sig[i];
            return ER_OK;
        }
    }
    return ER_ERR_NOT_FOUND;
}

int er_mix_particles(const er_structure* s, const er_forcefield* f, double eps_guest,
                     double sig_guest, er_particle* out, char* err, size_t errlen) {
    if (!s || !f || (s->n && !out)) return ER_ERR_INVALID;
    for (int i = 0; i < s->n; ++i) {
        out[i].x_f = s->x[i];
        out[i].y_f = s->y[i];
        out[i].z_f = s->z[i];
        double e = 0.0, sg = 0.0;
        if (er_forcefield_find(f, s->label[i].c_str(), &e, &sg) != ER_OK) {
            put_err(err, errlen, "Could not find framework atom " + s->label[i] +
                                     " in forcefield.");
            return ER_ERR_NOT_FOUND;
        }
        // src/load_fast_particle_f_array.h:35-36
        out[i].sig_with_adsorbate_squared = pow((sig_guest + sg) / 2.0, 2);
        out[i].eps_with_adsorbate = sqrt(eps_guest * e);
    }
    return ER_OK;
}

int er_adsorbate_mw(const char* root, const char* adsorbate, double* mw, char* err,
                    size_t errlen) {
    if (!adsorbate || !mw) return ER_ERR_INVALID;
    std::ifstream mf(join(root, "data/masses.def").c_str());
    if (mf.fail()) {
        put_err(err, errlen, "Masses file data/masses.def not present!");
        return ER_ERR_IO;
    }
    std::string line, label;
    getline(mf, line);
    double m = 0.0, found = -1.0;
    while (getline(mf, line)) {
        std::istringstream ls(line);
        ls >> label >> m;
        if (label == adsorbate) {
            found = m;
            break;
        }
    }
    if (found < 0.0) {
        put_err(err, errlen,
                std::string("No molecular weight for adsorbate ") + adsorbate +
                    " in data/masses.def");
        return ER_ERR_NOT_FOUND;
    }
    *mw = found;
    return ER_OK;
}

int er_read_uc(const char* root, const char* name, const char* which, int rep[3], char* err,
               size_t errlen) {
    if (!name || !which || !rep) return ER_ERR_INVALID;
    const std::string rel = std::string("data/uc_replications/") + name + "_" + which + ".uc";
    std::ifstream uc(join(root, rel).c_str());
    if (uc.fail()) {
        put_err(err, errlen, std::string("unit cell replication factor file not found in "
                                         "data/uc_replications/$frameworkname_") +
                                 which + ".uc");
        return ER_ERR_IO;
    }
    for (int k = 0; k < 3; ++k) {
        if (!(uc >> rep[k])) {
            put_err(err, errlen, "Problem reading UC file");
            return ER_ERR_IO;
        }
    }
    return ER_OK;
}

int er_write_uc(const char* root, const char* name, const char* which, const int rep[3]) {
    if (!name || !which || !rep) return ER_ERR_INVALID;
    const std::string rel = std::string("data/uc_replications/") + name + "_" + which + ".uc";
    FILE* fh = fopen(join(root, rel).c_str(), "w");
    if (!fh) return ER_ERR_IO;
    fprintf(fh, "%d %d %d\n", rep[0], rep[1], rep[2]);
    fclose(fh);
    return ER_OK;
}

int er_read_settings(const char* path, int kind, er_settings* s, char* err, size_t errlen) {
    if (!path || !s) return ER_ERR_INVALID;
    std::ifstream sim(path);
    if (sim.fail()) {
        put_err(err, errlen, "Simulation.input failed to open!");
        return ER_ERR_IO;
    }
    // defaults, src/readsettings.h:61-69 and :120-124
    memset(s, 0, sizeof(*s));
    snprintf(s->forcefield, sizeof(s->forcefield), "None");
    s->verbose = 0;
    s->grid_resolution = -1.0;
    snprintf(s->grid_output_format, sizeof(s->grid_output_format), "txt");
    s->r_cutoff_squared = 12.5 * 12.5;
    s->feynman_hibbs = 0;
    s->energy_threshold = 0.0;
    s->temperature = -1;
    s->insertions_per_a3 = -1;
    std::string word;
    while (sim >> word) {  // src/readsettings.h:73-92 / :128-141
        if (word == "Temperature") sim >> s->temperature;
        if (word == "VoidFractionEnergyThreshold") sim >> s->energy_threshold;
        if (word == "GridResolution") sim >> s->grid_resolution;
        if (word == "CutoffRadius") {
            sim >> s->r_cutoff_squared;
            s->r_cutoff_squared = s->r_cutoff_squared * s->r_cutoff_squared;
        }
        if (word == "Forcefield") {
            std::string v;
            sim >> v;
            snprintf(s->forcefield, sizeof(s->forcefield), "%s", v.c_str());
        }
        if (word == "GridOutputFormat") {
            std::string v;
            sim >> v;
            snprintf(s->grid_output_format, sizeof(s->grid_output_format), "%s", v.c_str());
        }
        if (word == "FeynmanHibbs") {
            bool b = false;
            sim >> b;
            s->feynman_hibbs = b;
        }
        if (word == "NumberOfInsertionsPerA3") sim >> s->insertions_per_a3;
        if (word == "verbosemode") {
            bool b = false;
            sim >> b;
            s->verbose = b;
        }
    }
    if (kind == ER_SETTINGS_GRID) {  // src/readsettings.h:95-106
        if (s->feynman_hibbs && s->temperature < 0.0) {
            put_err(err, errlen, "Missing Temperature in simulation.input");
            return ER_ERR_INVALID;
        }
        if (s->grid_resolution < 0.0) {
            put_err(err, errlen, "Missing GridResolution in simulation.input");
            return ER_ERR_INVALID;
        }
    } else if (kind == ER_SETTINGS_HENRY) {  // src/readsettings.h:144-155
        if (s->temperature < 0.0) {
            put_err(err, errlen, "Missing Temperature in simulation.input");
            return ER_ERR_INVALID;
        }
        if (s->insertions_per_a3 < 0.0) {
            put_err(err, errlen, "Missing NumberOfInsertionsPerA3 in simulation.input");
            return ER_ERR_INVALID;
        }
    }
    if (strcmp(s->forcefield, "None") == 0) {
        put_err(err, errlen, "Missing Forcefield in simulation.input");
        return ER_ERR_INVALID;
    }
    return ER_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ grid text files
namespace {

// Formats pencils [p0, p1) (pencil = (i, j), N_z values each) into `out`.
// mode 0: .txt (one line per pencil); mode 1: .cube (kJ/mol, 6 per line).
void format_pencils(const float* g, int nz, size_t p0, size_t p1, int mode, std::string& out) {
    char buf[64];
    out.clear();
    out.reserve((p1 - p0) * (size_t)nz * 14 + (p1 - p0) * 2);
    for (size_t p = p0; p < p1; ++p) {
        const float* row = g + p * (size_t)nz;
        int count = 0;
        for (int k = 0; k < nz; ++k) {
            double v = (double)row[k];
            if (mode == 1) v = v * 8.314 / 1000;
            const int n = snprintf(buf, sizeof(buf), "% 13.6E ", v);
            out.append(buf, (size_t)n);
            if (mode == 1) {
                if (++count == 6) {
                    out.push_back('\n');
                    count = 0;
                }
            }
        }
        out.push_back('\n');
    }
}

int write_pencils(FILE* fh, const float* g, int nx, int ny, int nz, int mode, int n_threads) {
    const size_t n_p = (size_t)nx * ny;
    int nth = n_threads > 0 ? n_threads : (int)std::max(1u, std::thread::hardware_concurrency());
    nth = (int)std::min<size_t>((size_t)nth, std::max<size_t>(n_p, 1));
    // bounded memory: at most ~256 MB of text in flight
    const size_t per_chunk =
        std::max<size_t>(1, (256u << 20) / std::max<size_t>((size_t)nz * 15, 1));
    std::vector<std::string> bufs(nth);
    for (size_t c0 = 0; c0 < n_p; c0 += per_chunk) {
        const size_t c1 = std::min(n_p, c0 + per_chunk);
        const size_t per = (c1 - c0 + nth - 1) / nth;
        std::vector<std::thread> th;
        for (int t = 0; t < nth; ++t) {
            const size_t a = std::min(c1, c0 + t * per), b = std::min(c1, a + per);
            th.emplace_back([=, &bufs]() { format_pencils(g, nz, a, b, mode, bufs[t]); });
        }
        for (auto& x : th) x.join();
        for (int t = 0; t < nth; ++t)
            if (!bufs[t].empty() && fwrite(bufs[t].data(), 1, bufs[t].size(), fh) != bufs[t].size())
                return ER_ERR_IO;
    }
    return ER_OK;
}

}  // namespace

extern "C" {

int er_write_grid_txt(const char* path, const float* grid, int nx, int ny, int nz,
                      int n_threads) {
    if (!path || !grid || nx < 1 || ny < 1 || nz < 1) return ER_ERR_INVALID;
    FILE* fh = fopen(path, "w");
    if (!fh) return ER_ERR_IO;
    fprintf(fh,
            "%d %d %d  = (N_x,N_y,N_z) grid points (grid is in fractional coords). Endpoints "
            "included.\n",
            nx, ny, nz);
    int st = write_pencils(fh, grid, nx, ny, nz, 0, n_threads);
    if (fclose(fh) != 0) st = ER_ERR_IO;
    return st;
}

int er_write_grid_cube(const char* path, const float* grid, int nx, int ny, int nz,
                       const double t[9], int n_threads) {
    if (!path || !grid || !t || nx < 2 || ny < 2 || nz < 2) return ER_ERR_INVALID;
    FILE* fh = fopen(path, "w");
    if (!fh) return ER_ERR_IO;
    // src/writegrid.cu:157-166
    fprintf(fh, "\nThis is a grid file.\n");
    fprintf(fh, "%d % 13.6lf % 13.6lf % 13.6lf\n", 0, 0.0, 0.0, 0.0);
    fprintf(fh, "%d % 13.6lf % 13.6lf % 13.6lf\n", nx, t[0] / (nx - 1), 0.0, 0.0);
    fprintf(fh, "%d % 13.6lf % 13.6lf % 13.6lf\n", ny, t[1] / (ny - 1), t[4] / (ny - 1), 0.0);
    fprintf(fh, "%d % 13.6lf % 13.6lf % 13.6lf\n", nz, t[2] / (nz - 1), t[5] / (nz - 1),
            t[8] / (nz - 1));
    int st = write_pencils(fh, grid, nx, ny, nz, 1, n_threads);
    if (fclose(fh) != 0) st = ER_ERR_IO;
    return st;
}

int er_read_grid_txt(const char* path, double* out, size_t cap, int dims[3], char* err,
                     size_t errlen) {
    if (!path || !dims) return ER_ERR_INVALID;
    std::ifstream gf(path);
    if (gf.fail()) {
        put_err(err, errlen, std::string("Grid file ") + path + " could not be loaded...");
        return ER_ERR_IO;
    }
    std::string line;
    getline(gf, line);
    std::istringstream hl(line);
    int nx = 0, ny = 0, nz = 0;
    hl >> nx >> ny >> nz;
    if (nx < 1 || ny < 1 || nz < 1) {
        put_err(err, errlen, "grid file header is not N_x N_y N_z");
        return ER_ERR_INVALID;
    }
    dims[0] = nx; dims[1] = ny; dims[2] = nz;
    const size_t n = (size_t)nx * ny * nz;
    if (!out) return ER_OK;  // dims query
    if (cap < n) {
        put_err(err, errlen, "output buffer too small");
        return ER_ERR_LIMIT;
    }
    // src/gcmc.cc:326-340: one z pencil per line, y faster than x
    int i = 0, j = 0;
    while (getline(gf, line)) {
        if (i >= nx) break;
        const char* p = line.c_str();
        for (int k = 0; k < nz; ++k) {
            char* end = nullptr;
            const double v = strtod(p, &end);
            if (end == p) {
                put_err(err, errlen, "grid file: short line");
                return ER_ERR_IO;
            }
            out[(size_t)k + (size_t)j * nz + (size_t)i * ny * nz] = v;
            p = end;
        }
        if (++j == ny) {
            ++i;
            j = 0;
        }
    }
    if (!(i == nx && j == 0)) {  // src/gcmc.cc:339-340
        put_err(err, errlen, "grid file: wrong number of lines");
        return ER_ERR_IO;
    }
    return ER_OK;
}

}  // extern "C"
