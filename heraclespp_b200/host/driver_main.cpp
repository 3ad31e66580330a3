// driver_main.cpp -- `heracles_b200 <file.ini> [options]`: the reference's
// executable (src/main.cpp) on the B200 path.  Reads the same .ini, builds
// the domain and the setup's initial state, runs the time loop on the device
// and prints the reference's summary lines (main.cpp:570-583).
//
// Options (the reference fixes these at CMake time, CMakeLists.txt:11-79):
//   --ndim=1|2|3  --geometry=Cartesian|Spherical  --gravity=Uniform|Point_mass|Internal_mass
//   --eos=PerfectGas|RadGas
//   --setup=<name>  --precision=fp64|fp32_mixed|fp64_fast  --device=N  --output=<file>
//   --output-dir=<dir> [--prefix=<name>]: outputs with the reference's dataset
//     set at its cadence (main.cpp:312-346, :357-385, :533-561): one at the
//     start when [Output] iter_frequency or time_frequency is set, then after
//     every step that reaches an output iteration or time, at t_end and at
//     max_iter (hcl_write_output: <dir>/<prefix>_<id>.hclraw and <prefix>.xmf).
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "heracles_b200.h"

namespace {

std::string opt_value(int argc, char** argv, const char* name, const char* def)
{
    const size_t len = std::strlen(name);
    for (int i = 2; i < argc; ++i) {
        if (std::strncmp(argv[i], name, len) == 0 && argv[i][len] == '=') {
            return std::string(argv[i] + len + 1);
        }
    }
    return def;
}

int die(const char* what, int rc)
{
    std::cerr << what << ": " << hcl_last_error() << '\n';
    return rc == HCL_OK ? EXIT_FAILURE : rc;
}

} // namespace

int main(int argc, char** argv)
{
    if (argc < 2) {
        std::cerr << "usage: heracles_b200 <path to the ini file> [options]\n";
        return EXIT_FAILURE;
    }
    hcl_build_options opt{};
    opt.ndim = std::atoi(opt_value(argc, argv, "--ndim", "0").c_str());
    const std::string geom = opt_value(argc, argv, "--geometry", "Cartesian");
    const std::string grav = opt_value(argc, argv, "--gravity", "Uniform");
    const std::string prec = opt_value(argc, argv, "--precision", "fp64");
    const std::string setup = opt_value(argc, argv, "--setup", "shock_tube");
    const std::string output = opt_value(argc, argv, "--output", "");
    const std::string outdir = opt_value(argc, argv, "--output-dir", "");
    const std::string prefix = opt_value(argc, argv, "--prefix", "result");
    opt.geometry = geom == "Spherical" ? HCL_GEOM_SPHERICAL : HCL_GEOM_CARTESIAN;
    opt.gravity = grav == "Point_mass"      ? HCL_GRAVITY_POINT_MASS
                  : grav == "Internal_mass" ? HCL_GRAVITY_INTERNAL_MASS
                                            : HCL_GRAVITY_UNIFORM;
    opt.precision = prec == "fp32_mixed" ? HCL_FP32_MIXED : (prec == "fp64_fast" ? HCL_FP64_FAST : HCL_FP64);
    opt.eos = opt_value(argc, argv, "--eos", "PerfectGas") == "RadGas" ? HCL_EOS_RAD_GAS : HCL_EOS_PERFECT_GAS;
    opt.device = std::atoi(opt_value(argc, argv, "--device", "0").c_str());
    opt.setup = setup.c_str();

    hcl_handle* h = nullptr;
    hcl_run_params run{};
    int rc = hcl_create_from_ini(argv[1], &opt, &h, &run);
    if (rc) {
        return die("setup", rc);
    }
    int n[3];
    int64_t ncells = 0;
    hcl_get_extents(h, n, &ncells);
    int nd = opt.ndim > 0 ? opt.ndim : (n[2] > 1 ? 3 : (n[1] > 1 ? 2 : 1));
    std::vector<double> sums(5, 0.0);
    hcl_conservation_sums(h, sums.data());
    const double initial_mass = sums[0];

    const auto start = std::chrono::steady_clock::now();
    hcl_run_result res{};
    if (outdir.empty()) {
        rc = hcl_run(h, &run, &res);
    } else {
        // the time loop in chunks that end where main() writes an output
        int output_id = -1, iter_output_id = -1, time_output_id = -1;
        int iter = 0;
        double t = 0.0;
        const double t_end = run.t_end;
        if (run.iter_frequency > 0 || run.time_frequency > 0) {
            ++iter_output_id;
            ++output_id;
            if ((rc = hcl_write_output(h, outdir.c_str(), prefix.c_str(), output_id, iter_output_id, time_output_id,
                                       iter, t))) {
                return die("output", rc);
            }
        }
        for (;;) {
            hcl_run_params p = run;
            p.iter_frequency = 0;
            p.time_frequency = 0.0;
            p.nsteps = 0;
            int next_iter = -1;
            double next_time = -1.0;
            if (run.iter_frequency > 0) {
                next_iter = (iter_output_id + 1) * run.iter_frequency;
                p.nsteps = std::max(1, next_iter - iter);
            }
            if (run.time_frequency > 0) {
                next_time = run.time_first_output + (time_output_id + 1) * run.time_frequency;
                p.t_end = std::min(t_end, next_time);
            }
            rc = hcl_run(h, &p, &res);
            if (rc) {
                break;
            }
            iter = res.iter;
            t = res.t;
            // the chunk ended on its own t_end (the dt of its last step was
            // clamped to it, main.cpp:366-378) or on max_iter
            const bool at_max = iter >= run.max_iter;
            const bool at_t = res.finished && !at_max;
            bool out = false;
            if (next_iter >= 0 && iter >= next_iter) {
                ++iter_output_id;
                out = true;
            }
            if (next_time >= 0 && at_t && p.t_end == next_time) {
                ++time_output_id;
                out = true;
            }
            const bool done = at_max || (at_t && p.t_end == t_end);
            if (out || done) {
                ++output_id;
                if ((rc = hcl_write_output(h, outdir.c_str(), prefix.c_str(), output_id, iter_output_id,
                                           time_output_id, iter, t))) {
                    return die("output", rc);
                }
            }
            if (done) {
                break;
            }
        }
    }
    const auto end = std::chrono::steady_clock::now();
    if (rc) {
        std::cerr << "Time = " << res.t << ", iteration = " << res.iter << ": " << hcl_last_error() << '\n';
        hcl_destroy(h);
        return EXIT_FAILURE;
    }
    hcl_conservation_sums(h, sums.data());
    const double final_mass = sums[0];
    int nx[3];
    hcl_get_interior(h, nx, nullptr);
    const double interior = (double)nx[0] * nx[1] * nx[2]; // main.cpp:571-574
    const double duration = std::chrono::duration<double>(end - start).count();
    std::cout << "Final time = " << res.t << " and number of iterations = " << res.iter << '\n';
    std::cout << "Mean performance: " << 1e-6 * res.iter * interior / duration << " Mcell-updates/s\n";
    std::cout << "Initial mass = " << initial_mass << " and change in mass = " << std::abs(initial_mass - final_mass)
              << '\n';
    if (!output.empty()) {
        std::vector<double> rho((size_t)ncells), rhou((size_t)ncells * nd), E((size_t)ncells);
        hcl_get_state(h, rho.data(), rhou.data(), E.data(), nullptr, HCL_HOST);
        std::ofstream f(output, std::ios::binary);
        const int32_t hdr[4] = {nd, n[0], n[1], n[2]};
        f.write(reinterpret_cast<const char*>(hdr), sizeof(hdr));
        f.write(reinterpret_cast<const char*>(&res.t), sizeof(double));
        f.write(reinterpret_cast<const char*>(rho.data()), (std::streamsize)(sizeof(double) * rho.size()));
        f.write(reinterpret_cast<const char*>(rhou.data()), (std::streamsize)(sizeof(double) * rhou.size()));
        f.write(reinterpret_cast<const char*>(E.data()), (std::streamsize)(sizeof(double) * E.size()));
    }
    std::cout << "--- End ---\n";
    hcl_destroy(h);
    return EXIT_SUCCESS;
}
