// bond_harmonic_b200.cu -- `bond_style harmonic/b200` for the reference GPUDPD executable:
// a Bond plugin (the reference's registry, src/force/bond.cuh:8-35) whose compute_force
// hands the reference's device buffers (positions, bond list, forces, per-bond energy,
// per-atom virial) to libdpd_b200's dpd_bond_compute_aos.  Same coefficients and
// contract as the stock harmonic style (src/force/bond_harmonic.cu:19-402).
#include "force/bond.cuh"
#include "shim_common.h"

class Bond_harmonic_b200 : public Bond {
    dpd_engine* eng = nullptr;

public:
    bool isEnabled(System& system) override
    {
        std::stringstream ss(system.input);
        std::string line;
        bool found = false;
        while (std::getline(ss, line)) {
            std::istringstream iss(line);
            std::string key, style, extra;
            iss >> key >> style;
            if (key == "bond_style" && style == "harmonic/b200") {
                if (iss >> extra) {
                    std::cout << "illegal bond_style harmonic/b200 command: " << line << std::endl;
                    exit(1);
                }
                found = true;
            }
        }
        if (!found) return false;
        eng = b200_engine(system, true, "bond_style harmonic/b200");
        return true;
    }

    void print_bond_info(System&) override
    {
        std::cout << "   bond forces computed by libdpd_b200 (" << dpd_version() << ")" << std::endl;
    }

    std::string getName() override { return "harmonic/b200"; }

    void compute_force(System& system, unsigned int step) override
    {
        Atoms& a = system.atoms;
        const bool log = step % system.run_p.log_f == 0;
        if (dpd_bond_compute_aos(eng, a.d_pos, a.d_bondlist, system.n_bonds, a.d_force, log ? a.d_bond_pe : nullptr,
                                 log ? a.d_viral : nullptr) != DPD_OK) {
            std::cout << "bond_style harmonic/b200: " << dpd_last_error(eng) << std::endl;
            exit(1);
        }
    }
};

REGISTER_BOND(Bond_harmonic_b200)
