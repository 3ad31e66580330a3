// capi_host.cpp -- host-only entry points of the C ABI: the .ini front end
// and the setup plugins.  Exceptions from the host layer are caught here and
// mapped to status codes (the reference's main catches them, main.cpp:594-604).
#include <cstdio>
#include <cstring>
#include <exception>
#include <stdexcept>
#include <string>
#include <vector>

#include "heracles_b200.h"
#include "ini_reader.hpp"
#include "param.hpp"
#include "setups.hpp"

namespace hcl::host {
int set_error(int code, std::string const& msg);
}

extern "C" {

int hcl_setup_initial_prim(const char* setup, const char* ini_path, int ndim, const int n_wg[3], int nghost,
                           const double* xc0, const double* xc1, const double* xc2, double* rho, double* u, double* P)
{
    using namespace hcl::host;
    if (!setup || !n_wg || !xc0 || !xc1 || !xc2 || !rho || !u || !P) {
        return set_error(HCL_ERR_ARGUMENT, "null argument");
    }
    try {
        INIReader reader = ini_path ? INIReader(ini_path) : INIReader::from_string("");
        if (reader.ParseError() < 0) {
            return set_error(HCL_ERR_CONFIG, std::string("cannot open ") + ini_path);
        }
        SetupGrid g{ndim, {n_wg[0], n_wg[1], n_wg[2]}, nghost, {xc0, xc1, xc2}};
        setup_initial_prim(setup, reader, g, rho, u, P);
    } catch (std::exception const& e) {
        return set_error(HCL_ERR_CONFIG, e.what());
    }
    return HCL_OK;
}

int hcl_create_from_ini(const char* ini_path, const hcl_build_options* opt, hcl_handle** out, hcl_run_params* run)
{
    using namespace hcl::host;
    if (!ini_path || !opt || !out) {
        return set_error(HCL_ERR_ARGUMENT, "null argument");
    }
    *out = nullptr;
    hcl_handle* h = nullptr;
    try {
        INIReader reader(ini_path);
        if (reader.ParseError() != 0) {
            return set_error(HCL_ERR_CONFIG, std::string("cannot parse ") + ini_path);
        }
        Param param(reader);
        int ndim = opt->ndim;
        if (ndim <= 0) {
            ndim = param.Nx_glob_ng[2] > 1 ? 3 : (param.Nx_glob_ng[1] > 1 ? 2 : 1);
        }
        hcl_config cfg = make_config(reader, param, ndim, opt->geometry, opt->gravity, opt->precision, opt->device);
        cfg.eos = opt->eos;
        int rc = hcl_create(&cfg, &h);
        if (rc) {
            return rc;
        }
        int n[3];
        int64_t N = 0;
        hcl_get_extents(h, n, &N);
        std::vector<double> xc[3];
        double* xcp[3];
        for (int d = 0; d < 3; ++d) {
            xc[d].assign(n[d], 0.0);
            xcp[d] = xc[d].data();
        }
        hcl_get_grid(h, nullptr, nullptr, xcp, nullptr, nullptr);
        std::vector<double> rho((size_t)N, 0.0), u((size_t)N * ndim, 0.0), P((size_t)N, 0.0);
        SetupGrid g{ndim, {n[0], n[1], n[2]}, cfg.nghost, {xcp[0], xcp[1], xcp[2]}};
        setup_initial_prim(opt->setup ? opt->setup : "shock_tube", reader, g, rho.data(), u.data(), P.data());
        if ((rc = hcl_set_state_from_prim(h, rho.data(), u.data(), P.data(), nullptr)) ||
            (rc = hcl_reset_clock(h, param.t_ini))) {
            hcl_destroy(h);
            return rc;
        }
        if (run) {
            std::memset(run, 0, sizeof(*run));
            run->cfl = param.cfl;
            run->t_end = param.t_end;
            run->max_iter = param.max_iter;
            run->iter_frequency = param.iter_output_frequency;
            run->time_frequency = param.time_output_frequency;
            run->time_first_output = param.time_first_output;
            run->nsteps = 0;
        }
    } catch (std::exception const& e) {
        if (h) {
            hcl_destroy(h);
        }
        return set_error(HCL_ERR_CONFIG, e.what());
    }
    *out = h;
    return HCL_OK;
}

} // extern "C"
