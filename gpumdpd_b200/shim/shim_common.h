// shim_common.h -- helpers shared by the b200 plugins of the reference executable
// (pair_style dpd/b200 and mdpd/b200, bond_style harmonic/b200, fix nve/b200): the run.in
// with the plugin styles renamed to the stock ones, and a libdpd_b200 engine built from
// the reference's System after its read_data (src/main/main.cu:29-33).
#pragma once
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "system/system.cuh"
#include "dpd_b200.h"

// The run.in text with every `/b200` style of a pair_style, bond_style or fix line renamed
// to the stock style, so the engine checks the reference's own grammar.  atomic: the
// engine sees atoms only (atom_style bond/angle become atomic).  bonded: atom_style angle
// becomes bond and the angle commands are dropped (the engine takes the bonds only).
static std::string b200_stock_text(const std::string& input, bool atomic)
{
    std::stringstream in(input), out;
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream iss(line);
        std::string key, a;
        iss >> key >> a;
        if (key == "pair_style" || key == "bond_style" || key == "fix") {
            size_t p;
            while ((p = line.find("/b200")) != std::string::npos) line.erase(p, 5);
        }
        if (key == "atom_style" && (a == "bond" || a == "angle")) line = atomic ? "atom_style atomic" : "atom_style bond";
        if (!atomic && (key == "angle_style" || key == "angle_coeff")) continue;
        out << line << "\n";
    }
    return out.str();
}

// A single-system engine for the reference's current System: box, types, masses (read
// back from the reference's __constant__ table), positions; its bonds when `bonded`.
static dpd_engine* b200_engine(System& system, bool bonded, const char* who)
{
    const int n = system.n_atoms;
    const int nt = system.n_atomtypes;
    std::vector<numtyp> mf(nt, (numtyp)1.0);
    if (cudaMemcpyFromSymbol(mf.data(), masses, sizeof(numtyp) * nt) != cudaSuccess) {
        std::cout << who << ": cannot read the masses" << std::endl;
        exit(1);
    }
    std::vector<double> x(3 * (size_t)n), v(3 * (size_t)n, 0.0), m(nt);
    for (int t = 0; t < nt; t++) m[t] = mf[t];
    std::vector<int> tag(n), type(n), mol;
    for (int i = 0; i < n; i++) {
        tag[i] = i + 1;  // rows are in tag order (index = id - 1)
        type[i] = system.atoms.h_type[i];
        for (int k = 0; k < 3; k++) x[3 * (size_t)i + k] = system.atoms.h_pos[3 * (size_t)i + k];
    }
    dpd_system s = {};
    s.n_atoms = n;
    s.n_atomtypes = nt;
    s.lo[0] = system.box.xlo; s.lo[1] = system.box.ylo; s.lo[2] = system.box.zlo;
    s.hi[0] = system.box.xhi; s.hi[1] = system.box.yhi; s.hi[2] = system.box.zhi;
    s.masses = m.data();
    s.tag = tag.data();
    s.type = type.data();
    s.x = x.data();
    s.v = v.data();
    if (bonded && system.atom_style != 0) {
        s.n_bonds = system.n_bonds;
        s.n_bondtypes = system.n_bondtypes;
        s.bonds = system.atoms.h_bondlist.data();
        mol = system.atoms.h_mol_id;
        if ((int)mol.size() == n) s.mol = mol.data();
    }
    const std::string text = b200_stock_text(system.input, !(bonded && system.atom_style != 0));
    dpd_engine* eng = nullptr;
    if (dpd_create_from_system(text.c_str(), &s, &eng) != DPD_OK) {
        std::cout << who << ": " << dpd_last_error(nullptr) << std::endl;
        exit(1);
    }
    return eng;
}
