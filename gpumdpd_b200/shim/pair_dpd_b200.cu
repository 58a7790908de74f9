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
#include "shim_common.h"

template <int STYLE>
class Pair_b200 : public Pair {
    dpd_engine* eng = nullptr;
    const char* name() const { return STYLE == 0 ? "dpd/b200" : "mdpd/b200"; }

public:
    bool isEnabled(System& system) override
    {
        // enabled when the run.in's pair_style names this style; the engine gets the same
        // text with the stock style names, so its grammar and checks are the reference's
        std::stringstream in(system.input);
        std::string line;
        bool found = false;
        while (std::getline(in, line)) {
            std::istringstream iss(line);
            std::string key, style;
            iss >> key >> style;
            if (key == "pair_style" && style == name()) found = true;
        }
        if (!found) return false;
        // bonds stay with the reference's bond style; the engine sees atoms only (masses do
        // not enter the pair force)
        eng = b200_engine(system, false, name());
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
