// fix_nve_b200.cu -- `fix ID group nve/b200` for the reference GPUDPD executable: a Fix
// plugin (the reference's registry, src/fix/fix.cuh:7-57; registered by name, since the
// style name is not an identifier) whose initial_integrate and final_integrate hand the
// reference's device buffers and the group's index list to libdpd_b200's dpd_nve_aos.
// Same contract as the stock nve (src/fix/fix_nve.cu:17-183).
#include "fix/fix.cuh"
#include "shim_common.h"

class Fix_nve_b200 : public Fix {
    dpd_engine* eng = nullptr;

    void integrate(System& system, int phase)
    {
        Group& g = find_group(system, group_id);
        Atoms& a = system.atoms;
        if (dpd_nve_aos(eng, phase, g.d_atoms, g.n_atoms, a.d_type, a.d_pos, a.d_uwpos, a.d_vel, a.d_force) != DPD_OK) {
            std::cout << "fix nve/b200: " << dpd_last_error(eng) << std::endl;
            exit(1);
        }
    }

public:
    Fix_nve_b200(std::string id, std::string gid, const std::vector<std::string>&) : Fix(id, gid) {}

    void validateParams(const std::vector<std::string>& params) override
    {
        if (!params.empty()) {
            std::cout << "illegal fix_nve/b200 command: fix ID groupID nve/b200" << std::endl;
            exit(1);
        }
    }

    std::string getName() override { return "nve/b200"; }

    void preprocess(System& system) override { eng = b200_engine(system, false, "fix nve/b200"); }

    void postprocess(System&) override
    {
        if (eng) dpd_destroy(eng);
        eng = nullptr;
    }

    void initial_integrate(System& system, unsigned int) override { integrate(system, 0); }
    void final_integrate(System& system, unsigned int) override { integrate(system, 1); }
};

static bool fix_nve_b200_registered = [] {
    registerFixType("nve/b200", [](const std::string& id, const std::string& gid,
                                   const std::vector<std::string>& params) -> std::unique_ptr<Fix> {
        return std::unique_ptr<Fix>(new Fix_nve_b200(id, gid, params));
    });
    return true;
}();
