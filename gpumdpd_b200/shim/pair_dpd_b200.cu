// pair_dpd_b200.cu -- `pair_style dpd/b200` and `pair_style mdpd/b200` for the reference
// GPUDPD executable: Pair plugins (the reference's own registry, src/force/pair.cuh:8-35)
// whose compute_force hands the reference's device buffers to libdpd_b200's
// dpd_pair_compute_aos.  Compiled into a copy of the reference's build together with its
// unmodified sources (oracle/build_ref.sh SHIM), it runs the reference's timestep loop --
// its integrator, bonds, thermo and dump -- with this engine computing the pair forces,
// which is the in-loop drop-in test of the boundary.  Needs -DSINGLE (float buffers).
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "force/pair.cuh"
#include "dpd_b200.h"

template <int STYLE>
class Pair_b200 : public Pair {
    dpd_engine* eng = nullptr;
    const char* name() const { return STYLE == 0 ? "dpd/b200" : "mdpd/b200"; }
    const char* stock() const { return STYLE == 0 ? "dpd" : "mdpd"; }

public:
    bool isEnabled(System& system) override
    {
        // enabled when the run.in's pair_style names this style; the engine gets the same
        // text with the stock style name, so its grammar and checks are the reference's
        std::stringstream in(system.input), out;
        std::string line;
        bool found = false;
        while (std::getline(in, line)) {
            std::istringstream iss(line);
            std::string key, style;
            iss >> key >> style;
            if (key == "pair_style" && style == name()) {
                found = true;
                std::string rest;
                std::getline(iss, rest);
                line = std::string("pair_style ") + stock() + rest;
            }
            out << line << "\n";
        }
        if (!found) return false;
        const int n = system.n_atoms;
        std::vector<double> x(3 * (size_t)n), v(3 * (size_t)n, 0.0), m(system.n_atomtypes, 1.0);
        std::vector<int> tag(n), type(n);
        for (int i = 0; i < n; i++) {
            tag[i] = i + 1;  // rows are in tag order (index = id - 1)
            type[i] = system.atoms.h_type[i];
            for (int k = 0; k < 3; k++) x[3 * (size_t)i + k] = system.atoms.h_pos[3 * (size_t)i + k];
        }
        dpd_system s = {};
        s.n_atoms = n;
        s.n_atomtypes = system.n_atomtypes;
        s.lo[0] = system.box.xlo; s.lo[1] = system.box.ylo; s.lo[2] = system.box.zlo;
        s.hi[0] = system.box.xhi; s.hi[1] = system.box.yhi; s.hi[2] = system.box.zhi;
        s.masses = m.data();  // masses do not enter the pair force
        s.tag = tag.data();
        s.type = type.data();
        s.x = x.data();
        s.v = v.data();
        // bonds stay with the reference's own bond style; the engine sees atoms only
        std::string text = out.str();
        for (const char* word : {"atom_style bond", "atom_style angle"}) {
            const size_t p = text.find(word);
            if (p != std::string::npos) text.replace(p, std::string(word).size(), "atom_style atomic");
        }
        if (dpd_create_from_system(text.c_str(), &s, &eng) != DPD_OK) {
            std::cout << "pair_style " << name() << ": " << dpd_last_error(nullptr) << std::endl;
            exit(1);
        }
        return true;
    }

    void print_pair_info(System&) override
    {
        std::cout << "   pair forces computed by libdpd_b200 (" << dpd_version() << ")" << std::endl;
    }

    std::string getName() override { return name(); }

    void compute_force(System& system, unsigned int step) override
    {
        Atoms& a = system.atoms;
        const bool log = step % system.run_p.log_f == 0;
        // the same contract as the stock styles: forces overwritten every step, per-atom PE
        // and virial on logged steps
        if (dpd_pair_compute_aos(eng, a.d_pos, a.d_vel, a.d_id, a.d_type, system.n_atoms, step, a.d_force,
                                 log ? a.d_pe : nullptr, log ? a.d_viral : nullptr) != DPD_OK) {
            std::cout << "pair_style " << name() << ": " << dpd_last_error(eng) << std::endl;
            exit(1);
        }
    }
};

using Pair_dpd_b200 = Pair_b200<0>;
using Pair_mdpd_b200 = Pair_b200<1>;
REGISTER_PAIR(Pair_dpd_b200)
REGISTER_PAIR(Pair_mdpd_b200)
