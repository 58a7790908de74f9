// main.cpp -- gpudpd_b200: drop-in replacement of the reference executable's driver
// (src/main/main.cu:15-72, src/main/utils.cuh:117-387).  Reads ./run.in, runs the
// timestep on the GPU through libdpd_b200.so, writes thermo.txt with the reference's
// columns (src/compute/thermo.cu:39-62,122-214), the data file of write_data, the
// all.trj frames of dump (src/system/dump.cu), the record file of fix spring and the
// files of the temp, rho, msd and tf computes.  `gpudpd_b200 --fp64 [run.in]` runs the
// FP64 parity engine instead, the counterpart of the reference's -DDOUBLE build (thermo.txt
// and write_data; the fixes, computes and dumps it does not cover are refused).
#include <chrono>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "dpd_b200.h"

int main(int argc, char** argv)
{
    bool fp64 = false;
    std::string path = "run.in";
    for (int k = 1; k < argc; k++) {
        if (std::string(argv[k]) == "--fp64") fp64 = true;
        else path = argv[k];
    }
    std::ifstream f(path);
    if (!f) {
        fprintf(stderr, "cannot open input file: %s\n", path.c_str());
        return 1;
    }
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string text = ss.str();
    auto t0 = std::chrono::steady_clock::now();
    dpd_engine* eng = nullptr;
    int e = fp64 ? dpd_create_fp64(text.c_str(), nullptr, nullptr, nullptr, &eng)
                 : dpd_create(text.c_str(), nullptr, nullptr, &eng);
    if (e) {
        fprintf(stderr, "ERROR: %s\n", dpd_last_error(nullptr));
        return 1;
    }
    // run, thermo and write_data settings are re-read from the text
    unsigned nsteps = 0;
    int atom_style = 0;
    std::string out_data, spring_file;
    bool dump = false;
    struct Comp { std::string id, style, file; };
    std::vector<Comp> comps;  // temp, rho, msd, tf, wall_contact computes and their files
    std::vector<std::string> cdumps;  // dump computes
    std::istringstream ls(text);
    std::string line;
    while (std::getline(ls, line)) {
        size_t h = line.find('#');
        if (h != std::string::npos) line = line.substr(0, h);
        std::istringstream t(line);
        std::string k, a;
        t >> k;
        if (k == "run") t >> nsteps;
        if (k == "atom_style") { t >> a; atom_style = a == "atomic" ? 0 : (a == "bond" ? 1 : 2); }
        if (k == "write_data") t >> out_data;
        if (k == "dump") dump = true;
        if (k == "compute") {
            std::vector<std::string> w;
            while (t >> a) w.push_back(a);
            if (w.size() >= 3 && (w[2] == "temp" || w[2] == "rho" || w[2] == "msd" || w[2] == "tf" ||
                                  w[2] == "wall_contact"))
                comps.push_back({w[0], w[2], w.back()});
            if (w.size() >= 3 && w[2] == "dump") cdumps.push_back(w[0]);
        }
        if (k == "fix") {
            // fix ID groupID spring k x y z r0 [file_name file_frequency]
            std::vector<std::string> w;
            while (t >> a) w.push_back(a);
            if (w.size() == 10 && w[2] == "spring") spring_file = w[8];
        }
    }
    // trajectory frames to all.trj with the run.in's dump settings (src/system/dump.cu:5-8)
    if (dump && dpd_dump_open(eng, "all.trj", 0, 0, 0)) {
        fprintf(stderr, "ERROR: %s\n", dpd_last_error(eng));
        dpd_destroy(eng);
        return 1;
    }
    for (const std::string& id : cdumps)
        if (dpd_compute_dump_open(eng, id.c_str(), nullptr)) {
            fprintf(stderr, "ERROR: %s\n", dpd_last_error(eng));
            dpd_destroy(eng);
            return 1;
        }
    e = dpd_run(eng, nsteps);
    if (!e && (dump || !cdumps.empty())) e = dpd_dump_close(eng);
    if (e) {
        fprintf(stderr, "ERROR: %s\n", dpd_last_error(eng));
        dpd_destroy(eng);
        return 1;
    }
    std::vector<dpd_thermo> rows(fp64 ? nsteps + 2 : 2048);
    int n = 0;
    dpd_get_thermo(eng, rows.data(), (int)rows.size(), &n);
    FILE* th = fopen("thermo.txt", "w");
    if (atom_style == 0)
        fprintf(th, "%15s\t%10s\t%20s\t%12s\t%12s\t%12s\t%12s\t%12s\t%12s\t%12s\n", "step", "temp", "pair_pe",
                "pressure", "pxx", "pxy", "pxz", "pyy", "pyz", "pzz");
    else if (atom_style == 1)
        fprintf(th, "%15s\t%10s\t%20s\t%20s\t%12s\t%12s\t%12s\t%12s\t%12s\t%12s\t%12s\n", "step", "temp",
                "pair_pe", "bond_pe", "pressure", "pxx", "pxy", "pxz", "pyy", "pyz", "pzz");
    else  // src/compute/thermo.cu:55-62
        fprintf(th, "%15s\t%10s\t%20s\t%20s\t%20s\t%12s\t%12s\t%12s\t%12s\t%12s\t%12s\t%12s\n", "step",
                "temp", "pair_pe", "bond_pe", "angle_pe", "pressure", "pxx", "pxy", "pxz", "pyy", "pyz", "pzz");
    for (int k = 0; k < n; k++) {
        const dpd_thermo& r = rows[k];
        if (atom_style == 0)
            fprintf(th, "%15lld\t%10.6f\t%20.6f\t%12.6f\t%12.6f\t%12.6f\t%12.6f\t%12.6f\t%12.6f\t%12.6f\n",
                    (long long)r.step, r.temp, r.pair_pe, r.pressure, r.p[0], r.p[1], r.p[2], r.p[3], r.p[4], r.p[5]);
        else if (atom_style == 1)
            fprintf(th, "%15lld\t%10.6f\t%20.6f\t%20.6f\t%12.6f\t%12.6f\t%12.6f\t%12.6f\t%12.6f\t%12.6f\t%12.6f\n",
                    (long long)r.step, r.temp, r.pair_pe, r.bond_pe, r.pressure, r.p[0], r.p[1], r.p[2], r.p[3],
                    r.p[4], r.p[5]);
        else
            fprintf(th,
                    "%15lld\t%10.6f\t%20.6f\t%20.6f\t%20.6f\t%12.6f\t%12.6f\t%12.6f\t%12.6f\t%12.6f\t%12.6f\t%12.6f\n",
                    (long long)r.step, r.temp, r.pair_pe, r.bond_pe, r.angle_pe, r.pressure, r.p[0], r.p[1], r.p[2],
                    r.p[3], r.p[4], r.p[5]);
    }
    fclose(th);
    if (!spring_file.empty()) {
        // src/fix/fix_spring.cu:118-128 (header) and 340-360 (rows)
        std::vector<double> sr(6 * 2048);
        int ns = 0;
        dpd_get_spring_records(eng, sr.data(), 2048, &ns);
        FILE* sf = fopen(spring_file.c_str(), "w");
        if (sf) {
            fprintf(sf, "%15s\t\t%15s\t\t%15s\t\t%15s\t\t%15s\t\t%15s\n", "step", "spring_force_x", "spring_force_y",
                    "spring_force_z", "spring_force", "spring_erergy");
            for (int k = 0; k < ns; k++) {
                const double* r = &sr[6 * (size_t)k];
                fprintf(sf, "%15lld\t\t%15g\t\t%15g\t\t%15g\t\t%15g\t\t%15g\n", (long long)r[0], r[1], r[2], r[3],
                        r[4], r[5]);
            }
            fclose(sf);
        }
    }
    // group compute files: src/compute/compute_temp.cu:34-40,160-170 and the same in
    // compute_rho.cu, compute_msd.cu, compute_tf.cu
    for (const Comp& c : comps) {
        std::vector<double> cr(4 * 2048);
        int nc = 0, nr = 0;
        if (dpd_get_compute(eng, c.id.c_str(), cr.data(), 2048, &nc, &nr)) continue;
        FILE* cf = fopen(c.file.c_str(), "w");
        if (!cf) continue;
        if (c.style == "tf")
            fprintf(cf, "%15s\t\t%15s\t\t%15s\t\t%15s\n", "step", "tf_x", "tf_y", "tf_z");
        else
            fprintf(cf, "%15s\t\t%15s\n", "step", c.style.c_str());
        for (int q = 0; q < nr; q++) {
            const double* r = &cr[(size_t)q * nc];
            fprintf(cf, "%15lld", (long long)r[0]);
            for (int j = 1; j < nc; j++) fprintf(cf, "\t\t%15g", r[j]);
            fprintf(cf, "\n");
        }
        fclose(cf);
    }
    if (!out_data.empty()) dpd_write_data(eng, out_data.c_str());
    int64_t natoms = 0;
    dpd_get_info(eng, nullptr, nullptr, &natoms, nullptr);
    dpd_destroy(eng);
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    double sps = (nsteps + 1) / secs;
    printf("   Performance:    %g steps/s    %g Matom*steps/s\n", sps, sps * natoms / 1e6);
    return 0;
}
