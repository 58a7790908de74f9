// dpd_io.cpp -- run.in grammar and data-file I/O of the reference, as code of this
// project.  The accepted commands, argument meanings and the checks that reject an
// input follow src/main/read_in.cu:40-371, src/force/pair_dpd.cu:19-173,
// src/force/pair_mdpd.cu:21-192, src/force/bond_harmonic.cu:19-147,
// src/system/system.cu:236-305 and src/fix/fix.cu:27-115; where the reference prints
// and calls exit(1), these functions return a negative status with the message.
#include "dpd_io.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <set>
#include <sstream>

#include "../../include/dpd_b200.h"

namespace dpd {

int tri_index(int ti, int tj, int nt)
{
    int a = ti < tj ? ti : tj, b = ti < tj ? tj : ti;
    return ((a - 1) * nt - (a - 1) * (a - 2) / 2 + b - a + 1) - 1;
}

static bool parse_double(const std::string& tok, double& out)
{
    try {
        size_t pos = 0;
        out = std::stod(tok, &pos);
        return pos > 0;
    } catch (...) {
        return false;
    }
}

// integers must be fully numeric, as parse_int in src/main/common.cuh:274-296
static bool parse_int(const std::string& tok, long long lo, long long hi, long long& out)
{
    try {
        size_t pos = 0;
        long long v = std::stoll(tok, &pos);
        if (pos != tok.size() || v < lo || v > hi) return false;
        out = v;
        return true;
    } catch (...) {
        return false;
    }
}

static int fail(std::string& err, const std::string& line, const std::string& what)
{
    err = what + (line.empty() ? "" : " (line: " + line + ")");
    return DPD_E_ARG;
}

int parse_run_in(const std::string& text, RunInput& in, std::string& err)
{
    static const std::set<std::string> allowed = {
        "atom_style", "neighbor", "timestep", "thermo", "run", "read_data", "write_data",
        "dump", "pair_style", "pair_coeff", "bond_style", "bond_coeff", "angle_style",
        "angle_coeff", "group", "fix", "compute"};
    bool got_atom_style = false, got_neighbor = false, got_timestep = false,
         got_thermo = false, got_run = false, got_read_data = false, got_pair_style = false,
         got_bond_style = false, got_angle_style = false;
    std::istringstream ss(text);
    std::string line;
    while (std::getline(ss, line)) {
        size_t hash = line.find('#');
        if (hash != std::string::npos) line = line.substr(0, hash);
        std::istringstream ls(line);
        std::vector<std::string> tok;
        std::string t;
        while (ls >> t) tok.push_back(t);
        if (tok.empty()) continue;
        const std::string key = tok[0];
        std::vector<std::string> args(tok.begin() + 1, tok.end());
        if (!allowed.count(key)) return fail(err, line, "unknown command " + key);
        in.lines.push_back(tok);
        in.raw.push_back(line);
        long long iv;
        if (key == "atom_style") {
            got_atom_style = true;
            if (args.size() != 1) return fail(err, line, "illegal atom_style command");
            if (args[0] == "atomic") in.atom_style = 0;
            else if (args[0] == "bond") in.atom_style = 1;
            else if (args[0] == "angle") in.atom_style = 2;
            else return fail(err, line, "illegal atom_style command");
        } else if (key == "neighbor") {
            got_neighbor = true;
            if (args.size() != 4) return fail(err, line, "illegal neighbor command");
            if (!parse_double(args[0], in.global_cut) || !parse_double(args[1], in.skin) ||
                !parse_double(args[2], in.max_rho) ||
                !parse_int(args[3], std::numeric_limits<int>::min(), std::numeric_limits<int>::max(), iv))
                return fail(err, line, "illegal neighbor command");
            in.nl_f = (int)iv;
            if (in.nl_f < 1) return fail(err, line, "neighbor check_frequency must be >= 1");
            if (in.global_cut <= 0 || in.skin < 0 || in.max_rho <= 0)
                return fail(err, line, "illegal neighbor command");
        } else if (key == "timestep") {
            got_timestep = true;
            if (args.size() != 1 || !parse_double(args[0], in.dt)) return fail(err, line, "illegal timestep command");
        } else if (key == "thermo") {
            got_thermo = true;
            if (args.size() != 1 || !parse_int(args[0], 0, 4294967295ll, iv)) return fail(err, line, "illegal thermo command");
            in.log_f = (unsigned)iv;
            if (in.log_f == 0) return fail(err, line, "thermo frequency must be >= 1");
        } else if (key == "run") {
            got_run = true;
            if (args.size() != 1 || !parse_int(args[0], 0, 4294967295ll, iv)) return fail(err, line, "illegal run command");
            in.nsteps = (unsigned)iv;
        } else if (key == "read_data") {
            got_read_data = true;
            if (args.size() != 1) return fail(err, line, "illegal read_data command");
            in.read_data = args[0];
        } else if (key == "write_data") {
            if (args.size() != 1) return fail(err, line, "illegal write_data command");
            in.write_data = true;
            in.write_data_name = args[0];
        } else if (key == "dump") {
            if (args.size() != 5) return fail(err, line, "illegal dump command");
            if (!parse_int(args[0], 0, 4294967295ll, iv)) return fail(err, line, "illegal dump command");
            in.dump_start = (unsigned)iv;
            if (!parse_int(args[1], 1, 4294967295ll, iv)) return fail(err, line, "illegal dump command");
            in.dump_f = (unsigned)iv;
            if (args[2] == "wrapped") in.dump_wrapped = true;
            else if (args[2] == "unwrapped") in.dump_wrapped = false;
            else return fail(err, line, "illegal dump command");
            if (args[3] == "force_yes") in.dump_force = true;
            else if (args[3] == "force_no") in.dump_force = false;
            else return fail(err, line, "illegal dump command");
            if (args[4] == "vel_yes") in.dump_vel = true;
            else if (args[4] == "vel_no") in.dump_vel = false;
            else return fail(err, line, "illegal dump command");
            in.dump = true;
        } else if (key == "pair_style") {
            got_pair_style = true;
        } else if (key == "bond_style") {
            got_bond_style = true;
        } else if (key == "angle_style") {
            got_angle_style = true;
        }
    }
    // required commands, in the order of Read_in::check (src/main/read_in.cu:294-371)
    if (!got_atom_style) return fail(err, "run.in", "atom_style command is missing");
    if (!got_neighbor) return fail(err, "run.in", "illegal neighbor command");
    if (!got_timestep) return fail(err, "run.in", "timestep command is missing");
    if (!got_thermo) return fail(err, "run.in", "thermo command is missing");
    if (!got_run) return fail(err, "run.in", "run command is missing");
    if (!got_read_data) return fail(err, "run.in", "read_data command is missing");
    if (!got_pair_style) return fail(err, "", "pair_style command is missing");
    if (in.atom_style == 1 && !got_bond_style) return fail(err, "", "bond_style command is missing");
    if (in.atom_style == 2) {
        if (!got_bond_style && !got_angle_style) return fail(err, "", "bond_style and angle_style commands are missing");
        if (!got_bond_style) return fail(err, "", "bond_style command is missing");
        if (!got_angle_style) return fail(err, "", "angle_style command is missing");
    }
    if (!(in.dt > 0)) return fail(err, "", "timestep must be > 0");
    return DPD_OK;
}

// ---------------------------------------------------------------------------------
// Data file reader.  Accepts the files written by src/system/read_data.cu:473-637 (and
// LAMMPS data files of the same layout); sections are found by keyword rather than
// by line position.  Positions are wrapped into the box on read
// (Read_data::adjust_coordinate, src/system/read_data.cu:192-197); atom index = id-1.

static bool starts_section(const std::string& l, const char* name)
{
    std::istringstream ls(l);
    std::string w;
    ls >> w;
    return w == name;
}

int read_data_file(const std::string& path, int atom_style, SystemData& s, std::string& err)
{
    std::ifstream f(path);
    if (!f) {
        err = "Cannot open data file: " + path;
        return DPD_E_IO;
    }
    std::vector<std::string> lines;
    std::string l;
    while (std::getline(f, l)) lines.push_back(l);
    size_t i = 1;  // first line is a comment
    bool box[3] = {false, false, false};
    // header
    for (; i < lines.size(); i++) {
        std::string h = lines[i];
        size_t hash = h.find('#');
        if (hash != std::string::npos) h = h.substr(0, hash);
        std::istringstream ls(h);
        std::vector<std::string> t;
        std::string w;
        while (ls >> w) t.push_back(w);
        if (t.empty()) continue;
        if (t[0] == "Masses" || t[0] == "Atoms" || t[0] == "Velocities" || t[0] == "Bonds" || t[0] == "Angles") break;
        long long iv;
        if (t.size() >= 2 && t[1] == "atoms" && parse_int(t[0], 0, 2147483647ll, iv)) s.n_atoms = (int)iv;
        else if (t.size() >= 2 && t[1] == "bonds" && parse_int(t[0], 0, 2147483647ll, iv)) s.n_bonds = (int)iv;
        else if (t.size() >= 2 && t[1] == "angles" && parse_int(t[0], 0, 2147483647ll, iv)) s.n_angles = (int)iv;
        else if (t.size() >= 3 && t[1] == "atom" && t[2] == "types" && parse_int(t[0], 0, 1000000, iv)) s.n_atomtypes = (int)iv;
        else if (t.size() >= 3 && t[1] == "bond" && t[2] == "types" && parse_int(t[0], 0, 1000000, iv)) s.n_bondtypes = (int)iv;
        else if (t.size() >= 3 && t[1] == "angle" && t[2] == "types" && parse_int(t[0], 0, 1000000, iv)) s.n_angletypes = (int)iv;
        else if (t.size() >= 4 && (t[2] == "xlo" || t[2] == "ylo" || t[2] == "zlo")) {
            int d = t[2] == "xlo" ? 0 : (t[2] == "ylo" ? 1 : 2);
            if (!parse_double(t[0], s.lo[d]) || !parse_double(t[1], s.hi[d])) {
                err = "Error reading box bounds from line: " + lines[i];
                return DPD_E_ARG;
            }
            box[d] = true;
        }
    }
    if (!box[0] || !box[1] || !box[2] || s.lo[0] >= s.hi[0] || s.lo[1] >= s.hi[1] || s.lo[2] >= s.hi[2]) {
        err = "Invalid box dimensions.";
        return DPD_E_ARG;
    }
    if (s.n_atoms <= 0 || s.n_atomtypes <= 0) {
        err = "data file header must give the numbers of atoms and atom types";
        return DPD_E_ARG;
    }
    s.type.assign(s.n_atoms, 0);
    s.mol.assign(s.n_atoms, 0);
    s.x.assign(3 * (size_t)s.n_atoms, 0.0);
    s.v.assign(3 * (size_t)s.n_atoms, 0.0);
    s.masses.assign(s.n_atomtypes, 0.0);
    std::vector<char> seen(s.n_atoms, 0), mass_seen(s.n_atomtypes, 0);
    bool got_atoms = false, got_masses = false, got_bonds = false, got_angles = false;
    auto next_rows = [&](size_t& k, int count, const std::function<bool(const std::vector<std::string>&)>& fn) -> bool {
        int done = 0;
        for (k++; k < lines.size() && done < count; k++) {
            std::string h = lines[k];
            size_t hash = h.find('#');
            if (hash != std::string::npos) h = h.substr(0, hash);
            std::istringstream ls(h);
            std::vector<std::string> t;
            std::string w;
            while (ls >> w) t.push_back(w);
            if (t.empty()) continue;
            if (!fn(t)) return false;
            done++;
        }
        k--;
        return done == count;
    };
    for (; i < lines.size(); i++) {
        const std::string& h = lines[i];
        if (starts_section(h, "Masses")) {
            bool ok = next_rows(i, s.n_atomtypes, [&](const std::vector<std::string>& t) {
                long long ty;
                double m;
                if (t.size() < 2 || !parse_int(t[0], 1, s.n_atomtypes, ty) || !parse_double(t[1], m)) return false;
                s.masses[ty - 1] = m;
                mass_seen[ty - 1] = 1;
                return true;
            });
            if (!ok) { err = "Error reading mass for atom type."; return DPD_E_ARG; }
            got_masses = true;
        } else if (starts_section(h, "Atoms")) {
            int file_style = atom_style;
            size_t hash = h.find('#');
            if (hash != std::string::npos) {
                std::istringstream ls(h.substr(hash + 1));
                std::string st;
                ls >> st;
                if (st == "atomic") file_style = 0;
                else if (st == "bond") file_style = 1;
                else if (st == "angle") file_style = 2;
                else { err = "Unknown atom_style in data file."; return DPD_E_ARG; }
            }
            if (file_style != atom_style) {
                err = "atom_style in run.in is inconsistent with the style in data file.";
                return DPD_E_ARG;
            }
            bool ok = next_rows(i, s.n_atoms, [&](const std::vector<std::string>& t) {
                size_t need = atom_style == 0 ? 5 : 6;
                if (t.size() < need) return false;
                long long id, ty, mol = 0;
                size_t o = 1;
                if (!parse_int(t[0], 1, s.n_atoms, id)) return false;
                if (atom_style != 0) {
                    if (!parse_int(t[1], std::numeric_limits<int>::min(), std::numeric_limits<int>::max(), mol)) return false;
                    o = 2;
                }
                if (!parse_int(t[o], 1, s.n_atomtypes, ty)) return false;
                double p[3];
                for (int d = 0; d < 3; d++)
                    if (!parse_double(t[o + 1 + d], p[d])) return false;
                size_t k = (size_t)(id - 1);
                if (seen[k]) return false;
                seen[k] = 1;
                s.type[k] = (int)ty;
                s.mol[k] = (int)mol;
                for (int d = 0; d < 3; d++) {
                    double L = s.hi[d] - s.lo[d];
                    double c = p[d];
                    if (!std::isfinite(c)) return false;
                    if (c >= s.hi[d] || c < s.lo[d]) c -= L * std::floor((c - s.lo[d]) / L);
                    if (c >= s.hi[d]) c = s.lo[d];
                    s.x[3 * k + d] = c;
                }
                return true;
            });
            if (!ok) { err = "Error reading the Atoms section (ids must be 1..N, each once)."; return DPD_E_ARG; }
            got_atoms = true;
        } else if (starts_section(h, "Velocities")) {
            std::vector<char> vseen(s.n_atoms, 0);
            bool ok = next_rows(i, s.n_atoms, [&](const std::vector<std::string>& t) {
                long long id;
                if (t.size() < 4 || !parse_int(t[0], 1, s.n_atoms, id)) return false;
                for (int d = 0; d < 3; d++)
                    if (!parse_double(t[1 + d], s.v[3 * (id - 1) + d])) return false;
                vseen[id - 1] = 1;
                return true;
            });
            if (!ok) { err = "Error reading the Velocities section."; return DPD_E_ARG; }
            s.has_velocities = true;
        } else if (starts_section(h, "Bonds")) {
            s.bonds.assign(3 * (size_t)s.n_bonds, -1);
            std::vector<char> bseen(s.n_bonds, 0);
            bool ok = next_rows(i, s.n_bonds, [&](const std::vector<std::string>& t) {
                long long id, ty, a, b;
                if (t.size() < 4 || !parse_int(t[0], 1, s.n_bonds, id) ||
                    !parse_int(t[1], 1, std::max(1, s.n_bondtypes), ty) ||
                    !parse_int(t[2], 1, s.n_atoms, a) || !parse_int(t[3], 1, s.n_atoms, b))
                    return false;
                if (bseen[id - 1] || a == b) return false;
                bseen[id - 1] = 1;
                s.bonds[3 * (id - 1)] = (int)ty;
                s.bonds[3 * (id - 1) + 1] = (int)a;
                s.bonds[3 * (id - 1) + 2] = (int)b;
                return true;
            });
            if (!ok) { err = "Error reading the Bonds section."; return DPD_E_ARG; }
            got_bonds = true;
        } else if (starts_section(h, "Angles")) {
            // src/system/read_data.cu:428-466: id type i j k, j the apex
            s.angles.assign(4 * (size_t)s.n_angles, -1);
            std::vector<char> aseen(s.n_angles, 0);
            bool ok = next_rows(i, s.n_angles, [&](const std::vector<std::string>& t) {
                long long id, ty, a, b, c;
                if (t.size() < 5 || !parse_int(t[0], 1, s.n_angles, id) ||
                    !parse_int(t[1], 1, std::max(1, s.n_angletypes), ty) ||
                    !parse_int(t[2], 1, s.n_atoms, a) || !parse_int(t[3], 1, s.n_atoms, b) ||
                    !parse_int(t[4], 1, s.n_atoms, c))
                    return false;
                if (aseen[id - 1] || a == b || b == c || a == c) return false;
                aseen[id - 1] = 1;
                s.angles[4 * (id - 1)] = (int)ty;
                s.angles[4 * (id - 1) + 1] = (int)a;
                s.angles[4 * (id - 1) + 2] = (int)b;
                s.angles[4 * (id - 1) + 3] = (int)c;
                return true;
            });
            if (!ok) { err = "Error reading the Angles section."; return DPD_E_ARG; }
            got_angles = true;
        }
    }
    if (!got_masses) { err = "Masses section is missing."; return DPD_E_ARG; }
    for (int t = 0; t < s.n_atomtypes; t++)
        if (!mass_seen[t] || !(s.masses[t] > 0)) { err = "All the masses are not set."; return DPD_E_ARG; }
    if (!got_atoms) { err = "Atoms section is missing."; return DPD_E_ARG; }
    if (atom_style >= 1 && s.n_bonds > 0 && !got_bonds) { err = "Bonds section is missing."; return DPD_E_ARG; }
    if (atom_style == 2 && s.n_angles > 0 && !got_angles) { err = "Angles section is missing."; return DPD_E_ARG; }
    if (atom_style == 0) s.n_bonds = 0;
    if (atom_style != 2) s.n_angles = 0;
    return DPD_OK;
}

// ---------------------------------------------------------------------------------
int parse_force_field(const RunInput& in, const SystemData& sys, ForceField& ff, std::string& err)
{
    const int nt = sys.n_atomtypes;
    ff.ntypes = nt;
    if (nt > 32) return fail(err, "", "at most 32 atom types are supported");
    const int npair = nt * (nt + 1) / 2;
    ff.coeff.assign(npair, {0, 0, 0, 0, 0});
    std::vector<char> got(npair, 0);
    int n_enabled = 0;
    // pair_style
    for (size_t k = 0; k < in.lines.size(); k++) {
        const auto& t = in.lines[k];
        const std::string& line = in.raw[k];
        if (t[0] != "pair_style") continue;
        if (t.size() < 2) return fail(err, line, "illegal pair_style command");
        long long iv;
        if (t[1] == "dpd") {
            n_enabled++;
            if (t.size() != 5) return fail(err, line, "illegal pair_style dpd command: pair_style dpd temp rc seed");
            if (!parse_double(t[2], ff.temp) || !parse_double(t[3], ff.rc) || !parse_int(t[4], 0, 4294967295ll, iv))
                return fail(err, line, "illegal pair_style dpd command: pair_style dpd temp rc seed");
            ff.seed = (unsigned)iv;
            ff.pair_style = 0;
            if (ff.rc > in.global_cut) return fail(err, line, "global rc should not be bigger than the global_cut (neighbor)");
        } else if (t[1] == "mdpd") {
            n_enabled++;
            if (t.size() != 6) return fail(err, line, "illegal pair_style mdpd command: pair_style mdpd temp rc rd seed");
            if (!parse_double(t[2], ff.temp) || !parse_double(t[3], ff.rc) || !parse_double(t[4], ff.rd) ||
                !parse_int(t[5], 0, 4294967295ll, iv))
                return fail(err, line, "illegal pair_style mdpd command: pair_style mdpd temp rc rd seed");
            ff.seed = (unsigned)iv;
            ff.pair_style = 1;
            if (ff.rc > in.global_cut) return fail(err, line, "global rc should not be bigger than the global_cut (neighbor)");
            if (ff.rd > ff.rc) return fail(err, line, "rd should not be bigger than rc");
        }
    }
    if (n_enabled > 1) return fail(err, "", "more than one enabled pair_style found");
    if (n_enabled == 0) return fail(err, "", "no enabled pair_style found");
    // pair_coeff
    for (size_t k = 0; k < in.lines.size(); k++) {
        const auto& t = in.lines[k];
        const std::string& line = in.raw[k];
        if (t[0] != "pair_coeff") continue;
        size_t na = t.size() - 1;
        long long ti, tj;
        double A = 0, B = 0, gamma = 0, rc = ff.rc, rd = ff.rd;
        if (ff.pair_style == 0) {
            // the reference accepts 4 or 6 arguments (rc in the 5th); 5 is accepted too
            if (na != 4 && na != 5 && na != 6) return fail(err, line, "illegal pair_coeff command for pair dpd: pair_coeff typei typej A gamma rc(optional)");
            if (!parse_int(t[1], std::numeric_limits<int>::min(), std::numeric_limits<int>::max(), ti) ||
                !parse_int(t[2], std::numeric_limits<int>::min(), std::numeric_limits<int>::max(), tj))
                return fail(err, line, "illegal pair_coeff command for pair dpd");
            if (ti > tj || tj > nt || ti < 1) return fail(err, line, "illegal pair_coeff command for pair dpd: typei <= typej");
            if (!parse_double(t[3], A) || !parse_double(t[4], gamma)) return fail(err, line, "illegal pair_coeff command for pair dpd");
            if (na >= 5 && !parse_double(t[5], rc)) return fail(err, line, "illegal pair_coeff command for pair dpd");
        } else {
            if (na != 5 && na != 7) return fail(err, line, "illegal pair_coeff command for pair mdpd: pair_coeff typei typej A B gamma rc(optional) rd(optional)");
            if (!parse_int(t[1], std::numeric_limits<int>::min(), std::numeric_limits<int>::max(), ti) ||
                !parse_int(t[2], std::numeric_limits<int>::min(), std::numeric_limits<int>::max(), tj))
                return fail(err, line, "illegal pair_coeff command for pair mdpd");
            if (ti > tj || tj > nt || ti < 1) return fail(err, line, "illegal pair_coeff command for pair mdpd: typei <= typej");
            if (!parse_double(t[3], A) || !parse_double(t[4], B) || !parse_double(t[5], gamma))
                return fail(err, line, "illegal pair_coeff command for pair mdpd");
            if (na == 7 && (!parse_double(t[6], rc) || !parse_double(t[7], rd)))
                return fail(err, line, "illegal pair_coeff command for pair mdpd");
            if (rd > rc) return fail(err, line, "rd should not be bigger than rc");
            if (!(rd > 0)) return fail(err, line, "rd must be > 0");
        }
        if (rc > in.global_cut) return fail(err, line, "global rc should not be bigger than the global_cut (neighbor)");
        if (!(rc > 0)) return fail(err, line, "rc must be > 0");
        if (gamma < 0) return fail(err, line, "gamma must be >= 0");
        int idx = tri_index((int)ti, (int)tj, nt);
        got[idx] = 1;
        ff.coeff[idx] = {A, B, gamma, rc, rd};
    }
    for (int p = 0; p < npair; p++)
        if (!got[p]) return fail(err, "", "all pair_coeff are not set");
    // bonds
    if (in.atom_style >= 1) {
        int nbs = 0;
        for (size_t k = 0; k < in.lines.size(); k++) {
            const auto& t = in.lines[k];
            if (t[0] != "bond_style") continue;
            if (t.size() < 2) return fail(err, in.raw[k], "illegal bond_style command");
            if (t[1] == "harmonic") ff.bond_style = 1;
            else if (t[1] == "fene") ff.bond_style = 2;
            else return fail(err, in.raw[k], "unknown bond_style " + t[1]);
            if (t.size() != 2) return fail(err, in.raw[k], "illegal bond_style command: bond_style harmonic");
            nbs++;
        }
        if (nbs != 1) return fail(err, "", "exactly one bond_style is required");
        int nbt = std::max(sys.n_bondtypes, 1);
        ff.bond_coeff.assign(nbt, {0, 0, 0, 0});
        std::vector<char> bgot(nbt, 0);
        for (size_t k = 0; k < in.lines.size(); k++) {
            const auto& t = in.lines[k];
            const std::string& line = in.raw[k];
            if (t[0] != "bond_coeff") continue;
            long long ty;
            size_t need = ff.bond_style == 1 ? 4 : 6;
            if (t.size() != need) return fail(err, line, ff.bond_style == 1 ? "illegal bond_coeff command for bond_style harmonic: bond_coeff type k r0" : "illegal bond_coeff command for bond_style fene: bond_coeff type K R0 epsilon sigma");
            if (!parse_int(t[1], 1, std::numeric_limits<int>::max(), ty)) return fail(err, line, "illegal bond_coeff command");
            if (ty > nbt) return fail(err, line, "type exceeds n_bond_types");
            std::array<double, 4> c = {0, 0, 0, 0};
            for (size_t q = 2; q < need; q++)
                if (!parse_double(t[q], c[q - 2])) return fail(err, line, "illegal bond_coeff command");
            if (ff.bond_style == 2 && !(c[1] > 0)) return fail(err, line, "fene R0 must be > 0");
            ff.bond_coeff[ty - 1] = c;
            bgot[ty - 1] = 1;
        }
        for (int b = 0; b < sys.n_bondtypes; b++)
            if (!bgot[b]) return fail(err, "", "all bond_coeff are not set");
    }
    // angles, src/force/angle_harmonic.cu:19-147 (angle_style harmonic; angle_coeff type k theta0)
    if (in.atom_style == 2) {
        int nas = 0;
        for (size_t k = 0; k < in.lines.size(); k++) {
            const auto& t = in.lines[k];
            if (t[0] != "angle_style") continue;
            if (t.size() != 2) return fail(err, in.raw[k], "illegal angle_style harmonic command: angle_style angle_style");
            if (t[1] != "harmonic") return fail(err, in.raw[k], "unknown angle_style " + t[1]);
            ff.angle_style = 1;
            nas++;
        }
        if (nas != 1) return fail(err, "", "exactly one angle_style is required");
        int nat = std::max(sys.n_angletypes, 1);
        ff.angle_coeff.assign(nat, {0, 0});
        std::vector<char> agot(nat, 0);
        for (size_t k = 0; k < in.lines.size(); k++) {
            const auto& t = in.lines[k];
            const std::string& line = in.raw[k];
            if (t[0] != "angle_coeff") continue;
            long long ty;
            if (t.size() != 4) return fail(err, line, "illegal angle_coeff command for angle_style harmonic: angle_coeff type k theta0");
            if (!parse_int(t[1], 1, std::numeric_limits<int>::max(), ty)) return fail(err, line, "illegal angle_coeff command for angle_style harmonic");
            if (ty > nat) return fail(err, line, "type exceeds n_angle_types");
            std::array<double, 2> c = {0, 0};
            if (!parse_double(t[2], c[0]) || !parse_double(t[3], c[1]))
                return fail(err, line, "illegal angle_coeff command for angle_style harmonic");
            ff.angle_coeff[ty - 1] = c;
            agot[ty - 1] = 1;
        }
        for (int a = 0; a < sys.n_angletypes; a++)
            if (!agot[a]) return fail(err, "", "all angle_coeff are not set");
    }
    // groups, src/system/system.cu:236-305
    for (size_t k = 0; k < in.lines.size(); k++) {
        const auto& t = in.lines[k];
        const std::string& line = in.raw[k];
        if (t[0] != "group") continue;
        if (t.size() < 4 || t[2] != "type") return fail(err, line, "illegal group command: group group_name type type1 type2 ...");
        if (ff.groups.count(t[1])) return fail(err, line, "Group " + t[1] + " already exists");
        std::vector<int> types;
        std::set<int> tset;
        for (size_t q = 3; q < t.size(); q++) {
            long long ty;
            if (!parse_int(t[q], 1, std::numeric_limits<int>::max(), ty)) return fail(err, line, "illegal group command");
            if (ty > nt) return fail(err, line, "Type in group is not included in the data file");
            if (tset.count((int)ty)) return fail(err, line, "Duplicate type found: " + std::to_string(ty));
            tset.insert((int)ty);
            types.push_back((int)ty);
        }
        ff.groups[t[1]] = types;
    }
    // fixes, src/fix/fix.cu:27-115: nve, and the group fixes spring, rvcm and recenter
    // (validateParams of src/fix/fix_spring.cu:17-52, fix_rvcm.cu:17-40, fix_recenter.cu:17-32)
    std::set<std::string> fix_ids;
    auto group_mask = [&](const std::string& g) {
        uint32_t m = 0;
        for (int ty : ff.groups[g]) m |= 1u << (ty - 1);
        return m;
    };
    for (size_t k = 0; k < in.lines.size(); k++) {
        const auto& t = in.lines[k];
        const std::string& line = in.raw[k];
        if (t[0] != "fix") continue;
        if (t.size() < 4) return fail(err, line, "illegal fix command: fix ID groupID style params");
        if (fix_ids.count(t[1])) return fail(err, line, "Fix ID '" + t[1] + "' is already registered!");
        fix_ids.insert(t[1]);
        if (!ff.groups.count(t[2])) return fail(err, line, "Group '" + t[2] + "' not found!");
        const size_t np = t.size() - 4;
        if (t[3] == "spring") {
            const char* msg = "illegal fix_spring command: fix ID groupID spring spring_k spring_x spring_y spring_z spring_r0 file_name(optional) file_frequency(optional)";
            if (np != 5 && np != 7) return fail(err, line, msg);
            if (ff.spring.on) return fail(err, line, "this engine takes at most one fix spring");
            double v[5];
            for (int q = 0; q < 5; q++)
                if (!parse_double(t[4 + q], v[q])) return fail(err, line, msg);
            long long fq = 0;
            if (np == 7 && !parse_int(t[10], 1, 4294967295ll, fq)) return fail(err, line, msg);
            const char* axis[3] = {"x", "y", "z"};
            for (int d = 0; d < 3; d++)
                if (v[1 + d] < sys.lo[d] || v[1 + d] > sys.hi[d])
                    return fail(err, line, std::string("spring position is out of the box in ") + axis[d] + " direction!");
            ff.spring.on = true;
            ff.spring.mask = group_mask(t[2]);
            ff.spring.k = v[0];
            for (int d = 0; d < 3; d++) ff.spring.c[d] = v[1 + d];
            ff.spring.r0 = v[4];
            if (np == 7) {
                ff.spring.file = t[9];
                ff.spring.file_freq = (unsigned)fq;
            }
            continue;
        }
        if (t[3] == "rvcm") {
            const char* msg = "illegal fix_rvcm command: fix ID groupID rvcm frequency x_flag(0/1) y_flag(0/1) z_flag(0/1)";
            if (np != 4) return fail(err, line, msg);
            if (ff.rvcm.on) return fail(err, line, "this engine takes at most one fix rvcm");
            long long fq, fl[3];
            if (!parse_int(t[4], 1, 4294967295ll, fq)) return fail(err, line, msg);
            for (int d = 0; d < 3; d++)
                if (!parse_int(t[5 + d], 0, 1, fl[d])) return fail(err, line, msg);
            ff.rvcm.on = true;
            ff.rvcm.mask = group_mask(t[2]);
            ff.rvcm.freq = (unsigned)fq;
            for (int d = 0; d < 3; d++) ff.rvcm.flag[d] = (int)fl[d];
            continue;
        }
        if (t[3] == "recenter") {
            const char* msg = "illegal fix_recenter command: fix ID groupID recenter frequency recenter_x recenter_y recenter_z";
            if (np != 4) return fail(err, line, msg);
            if (ff.recenter.on) return fail(err, line, "this engine takes at most one fix recenter");
            long long fq;
            if (!parse_int(t[4], 1, 4294967295ll, fq)) return fail(err, line, msg);
            double c[3];
            for (int d = 0; d < 3; d++)
                if (!parse_double(t[5 + d], c[d])) return fail(err, line, msg);
            // src/fix/fix_recenter.cu:84-100 (its messages name the spring)
            const char* axis[3] = {"x", "y", "z"};
            for (int d = 0; d < 3; d++)
                if (c[d] < sys.lo[d] || c[d] > sys.hi[d])
                    return fail(err, line, std::string("spring position is out of the box in ") + axis[d] + " direction!");
            ff.recenter.on = true;
            ff.recenter.mask = group_mask(t[2]);
            ff.recenter.freq = (unsigned)fq;
            for (int d = 0; d < 3; d++) ff.recenter.c[d] = c[d];
            continue;
        }
        auto direction = [](const std::string& s) { return s == "x" ? 0 : (s == "y" ? 1 : (s == "z" ? 2 : -1)); };
        if (t[3] == "move") {
            // src/fix/fix_move.cu:17-30
            const char* msg = "illegal fix_move command: fix ID groupID move v_x v_y v_z";
            FixMove m;
            if (np != 3) return fail(err, line, msg);
            for (int d = 0; d < 3; d++)
                if (!parse_double(t[4 + d], m.v[d])) return fail(err, line, msg);
            if (ff.moves.size() >= 4) return fail(err, line, "this engine takes at most 4 fix move");
            m.mask = group_mask(t[2]);
            ff.moves.push_back(m);
            continue;
        }
        if (t[3] == "wall_reflect") {
            // src/fix/fix_wall_reflect.cu:17-45 and the in-box check of :50-80
            const char* msg = "illegal fix_wall_reflect command: fix ID groupID wall_reflect lo_wall_pos hi_wall_pos wall_direction";
            FixWallReflect w;
            if (np != 3 || !parse_double(t[4], w.lo) || !parse_double(t[5], w.hi)) return fail(err, line, msg);
            if (w.lo >= w.hi) return fail(err, line, std::string(msg) + ": lo_wall_pos should lower than hi_wall_pos");
            w.dir = direction(t[6]);
            if (w.dir < 0) return fail(err, line, std::string(msg) + ": Invalid fix_wall_reflect direction");
            if (w.lo < sys.lo[w.dir] || w.hi > sys.hi[w.dir]) return fail(err, line, "Wall position is out of the box!");
            if (ff.reflects.size() >= 4) return fail(err, line, "this engine takes at most 4 fix wall_reflect");
            w.mask = group_mask(t[2]);
            ff.reflects.push_back(w);
            continue;
        }
        if (t[3] == "two_wall") {
            // src/fix/fix_two_wall.cu:17-40
            const char* msg = "illegal fix_two_wall command: fix ID groupID two_wall lo_wall_name hi_wall_name direction";
            FixTwoWall w;
            if (np != 3) return fail(err, line, msg);
            for (int q = 4; q <= 5; q++)
                if (!ff.groups.count(t[q])) return fail(err, line, "Group '" + t[q] + "' not found!");
            w.dir = direction(t[6]);
            if (w.dir < 0) return fail(err, line, std::string(msg) + ": Invalid fix_two_wall direction");
            if (ff.twowalls.size() >= 2) return fail(err, line, "this engine takes at most 2 fix two_wall");
            w.mask = group_mask(t[2]);
            w.lo_mask = group_mask(t[4]);
            w.hi_mask = group_mask(t[5]);
            ff.twowalls.push_back(w);
            continue;
        }
        if (t[3] != "nve")
            return fail(err, line, "Fix type '" + t[3] + "' not found! (this engine implements nve, spring, rvcm, recenter, "
                                   "move, wall_reflect, two_wall)");
        if (t.size() != 4) return fail(err, line, "illegal fix_nve command: fix ID groupID nve");
        for (int ty : ff.groups[t[2]]) {
            uint32_t bit = 1u << (ty - 1);
            if (ff.integ_mask & bit) return fail(err, line, "type " + std::to_string(ty) + " is integrated by two nve fixes");
            ff.integ_mask |= bit;
        }
    }
    // computes, src/compute/compute.cu:60-115: temp, rho, msd, tf (per group) and rdf (new)
    std::set<std::string> cids;
    for (size_t k = 0; k < in.lines.size(); k++) {
        const auto& t = in.lines[k];
        const std::string& line = in.raw[k];
        if (t[0] != "compute") continue;
        if (t.size() < 4) return fail(err, line, "illegal compute command: compute ID groupID style params");
        if (cids.count(t[1])) return fail(err, line, "Compute ID '" + t[1] + "' is already registered!");
        cids.insert(t[1]);
        if (!ff.groups.count(t[2])) return fail(err, line, "Group '" + t[2] + "' not found!");
        long long iv;
        if (t[3] == "temp" || t[3] == "msd" || t[3] == "tf" || t[3] == "rho") {
            // validateParams of src/compute/compute_temp.cu:17-30, compute_msd.cu:17-30,
            // compute_tf.cu:17-30, compute_rho.cu:17-37; region checks of compute_rho.cu:42-75
            const bool rho = t[3] == "rho";
            const std::string msg = "illegal compute_" + t[3] + " command: compute ID groupID " + t[3] +
                                    (rho ? " frequency xlo xhi ylo yhi zlo zhi filename" : " frequency filename");
            if (t.size() != (rho ? 12u : 6u) || !parse_int(t[4], 1, 4294967295ll, iv)) return fail(err, line, msg);
            GroupCompute c;
            c.id = t[1];
            c.group = t[2];
            c.kind = t[3] == "temp" ? GC_TEMP : (t[3] == "msd" ? GC_MSD : (t[3] == "tf" ? GC_TF : GC_RHO));
            c.frequency = (unsigned)iv;
            c.file = t.back();
            for (int ty : ff.groups[t[2]]) c.type_mask |= 1u << (ty - 1);
            if (rho) {
                for (int q = 0; q < 6; q++)
                    if (!parse_double(t[5 + q], c.region[q])) return fail(err, line, msg);
                const char* nm[3] = {"x", "y", "z"};
                for (int d = 0; d < 3; d++) {
                    if (c.region[2 * d] < sys.lo[d])
                        return fail(err, line, msg + ": " + nm[d] + "lo < box." + nm[d] + "lo");
                    if (c.region[2 * d + 1] > sys.hi[d])
                        return fail(err, line, msg + ": " + nm[d] + "hi > box." + nm[d] + "hi");
                }
            }
            if (ff.gcs.size() >= 4) return fail(err, line, "this engine takes at most 4 temp/rho/msd/tf computes");
            ff.gcs.push_back(c);
        } else if (t[3] == "dump") {
            // src/compute/compute_dump.cu:17-30
            if (t.size() != 6 || !parse_int(t[4], 1, 4294967295ll, iv))
                return fail(err, line, "illegal compute_dump command: compute ID groupID dump frequency filename");
            ComputeDump c;
            c.id = t[1];
            c.frequency = (unsigned)iv;
            c.file = t[5];
            for (int ty : ff.groups[t[2]]) c.mask |= 1u << (ty - 1);
            ff.cdumps.push_back(c);
        } else if (t[3] == "wall_contact") {
            // src/compute/compute_wall_contact.cu:17-45
            const std::string msg = "illegal compute_wall_contact command: compute ID groupID wall_contact frequency "
                                    "wall_groupname lo/hi wall_direction cutoff filename";
            GroupCompute c;
            if (t.size() != 10 || !parse_int(t[4], 1, 4294967295ll, iv)) return fail(err, line, msg);
            if (!ff.groups.count(t[5])) return fail(err, line, "Group '" + t[5] + "' not found!");
            if (t[6] != "lo" && t[6] != "hi") return fail(err, line, msg);
            c.wall_dir = t[7] == "x" ? 0 : (t[7] == "y" ? 1 : (t[7] == "z" ? 2 : -1));
            if (c.wall_dir < 0 || !parse_double(t[8], c.cutoff)) return fail(err, line, msg);
            c.id = t[1];
            c.group = t[2];
            c.kind = GC_WALL;
            c.frequency = (unsigned)iv;
            c.file = t[9];
            c.wall_side = t[6] == "lo" ? 1 : -1;
            for (int ty : ff.groups[t[2]]) c.type_mask |= 1u << (ty - 1);
            for (int ty : ff.groups[t[5]]) c.wall_mask |= 1u << (ty - 1);
            if (ff.gcs.size() >= 4) return fail(err, line, "this engine takes at most 4 temp/rho/msd/tf/wall_contact computes");
            ff.gcs.push_back(c);
        } else if (t[3] == "rdf") {
            // compute ID groupID rdf typeA typeB rmax nbins every filename
            ComputeRdf c;
            long long a, b, nb, ev;
            if (t.size() != 10 || !parse_int(t[4], 1, nt, a) || !parse_int(t[5], 1, nt, b) ||
                !parse_double(t[6], c.rmax) || !parse_int(t[7], 1, 512, nb) ||
                !parse_int(t[8], 1, 1000000000ll, ev))
                return fail(err, line, "illegal compute_rdf command: compute ID groupID rdf typeA typeB rmax nbins every filename");
            c.id = t[1];
            c.ta = (int)a;
            c.tb = (int)b;
            c.nbins = (int)nb;
            c.every = (int)ev;
            c.file = t[9];
            if (!(c.rmax > 0)) return fail(err, line, "rdf rmax must be > 0");
            if (!ff.rdfs.empty()) return fail(err, line, "only one rdf compute is supported");
            ff.rdfs.push_back(c);
        } else {
            return fail(err, line, "Compute type '" + t[3] + "' not found! (this engine implements temp, rho, msd, tf, wall_contact, dump and rdf)");
        }
    }
    return DPD_OK;
}

// Data file writer in the reference's write_data layout (src/system/read_data.cu:473-637).
int write_data_file(const std::string& path, int atom_style, const SystemData& s, std::string& err)
{
    FILE* f = fopen(path.c_str(), "w");
    if (!f) {
        err = "Error opening file: " + path;
        return DPD_E_IO;
    }
    fprintf(f, "# Lammps format data file\n");
    fprintf(f, "                         \n");
    fprintf(f, "%d atoms\n", s.n_atoms);
    if (atom_style >= 1) fprintf(f, "%d bonds\n", s.n_bonds);
    if (atom_style == 2) fprintf(f, "%d angles\n", s.n_angles);
    fprintf(f, "%d atom types\n", s.n_atomtypes);
    if (atom_style >= 1) fprintf(f, "%d bond types\n", s.n_bondtypes);
    if (atom_style == 2) fprintf(f, "%d angle types\n", s.n_angletypes);
    fprintf(f, "                           \n");
    fprintf(f, "%.9f %.9f xlo xhi\n", s.lo[0], s.hi[0]);
    fprintf(f, "%.9f %.9f ylo yhi\n", s.lo[1], s.hi[1]);
    fprintf(f, "%.9f %.9f zlo zhi\n", s.lo[2], s.hi[2]);
    fprintf(f, "                           \n");
    fprintf(f, "Masses\n");
    fprintf(f, "                           \n");
    for (int t = 0; t < s.n_atomtypes; t++) fprintf(f, "%d %.9f\n", t + 1, s.masses[t]);
    fprintf(f, "                           \n");
    fprintf(f, atom_style == 0 ? "Atoms  # atomic\n" : (atom_style == 1 ? "Atoms  # bond\n" : "Atoms  # angle\n"));
    fprintf(f, "                           \n");
    for (int i = 0; i < s.n_atoms; i++) {
        if (atom_style >= 1)
            fprintf(f, "%d %d %d %.9f %.9f %.9f\n", i + 1, s.mol.empty() ? 0 : s.mol[i], s.type[i],
                    s.x[3 * i], s.x[3 * i + 1], s.x[3 * i + 2]);
        else
            fprintf(f, "%d %d %.9f %.9f %.9f\n", i + 1, s.type[i], s.x[3 * i], s.x[3 * i + 1], s.x[3 * i + 2]);
    }
    fprintf(f, "                           \n");
    fprintf(f, "Velocities\n");
    fprintf(f, "                           \n");
    for (int i = 0; i < s.n_atoms; i++)
        fprintf(f, "%d %.9f %.9f %.9f\n", i + 1, s.v[3 * i], s.v[3 * i + 1], s.v[3 * i + 2]);
    fprintf(f, "                           \n");
    if (atom_style >= 1) {
        fprintf(f, "Bonds\n");
        fprintf(f, "                           \n");
        for (int b = 0; b < s.n_bonds; b++)
            fprintf(f, "%d %d %d %d\n", b + 1, s.bonds[3 * b], s.bonds[3 * b + 1], s.bonds[3 * b + 2]);
    }
    if (atom_style == 2) {
        fprintf(f, "                           \n");
        fprintf(f, "Angles\n");
        fprintf(f, "                           \n");
        for (int a = 0; a < s.n_angles; a++)
            fprintf(f, "%d %d %d %d %d\n", a + 1, s.angles[4 * a], s.angles[4 * a + 1], s.angles[4 * a + 2],
                    s.angles[4 * a + 3]);
    }
    fclose(f);
    return DPD_OK;
}

}  // namespace dpd
