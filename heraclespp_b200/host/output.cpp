// output.cpp -- outputs and restarts with the reference's dataset set.
//
// The reference writes each output as an HDF5 file through PDI
// (io/io.cpp:185-318, datasets of io/config.yaml.cpp:7-265) and restarts from
// one (read_pdi, io/io.cpp:326-420; main.cpp:225-246).  This image has no HDF5
// library, so the same datasets go into a raw container:
//
//   "HCLRAW01"                      8 bytes
//   index length L                  uint64, little endian
//   index                           L bytes of text, one line per dataset:
//                                   "<name> <f64|i32> <byte offset> <rank> <extents...>"
//                                   (extents slowest first, as in the HDF5 files)
//   data                            little-endian values at 64-byte aligned offsets
//
// Scalars: output_id, iter_output_id, time_output_id, iter (i32), current_time,
// gamma (f64).  Nodes: x0..x2 with ghosts (n_wg + 1), x0_ng..x2_ng interior
// (nx + 1).  Cell fields over the interior in C order [nx2][nx1][nx0]: rho,
// ux0..ux{ndim-1}, P, E, T, fx0..fx{nfx-1}.  E is the conservative energy
// main() holds; u, P and T come from conv_cons_to_prim and temperature() over
// the current state (hcl_get_prim).
//
// "<prefix>.xmf" is rewritten at each output with every output of the run so
// far, a temporal collection of 3-D rectilinear grids whose attributes are
// Binary data items pointing into the raw files (the structure of the
// reference's XmlWriter, io/io.hpp:56-81, over raw files instead of HDF5).
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "heracles_b200.h"

namespace hcl::host {
int set_error(int code, std::string const& msg);
}

namespace {

using hcl::host::set_error;

constexpr char kMagic[9] = "HCLRAW01";

struct Dataset {
    std::string name;
    bool f64 = true;
    std::vector<int64_t> ext; // slowest first
    std::vector<double> d;
    std::vector<int32_t> i;
    uint64_t offset = 0;
    size_t bytes() const { return f64 ? d.size() * 8 : i.size() * 4; }
};

std::string file_name(const std::string& prefix, int output_id)
{
    char buf[32];
    std::snprintf(buf, sizeof(buf), "_%08d.hclraw", output_id);
    return prefix + buf;
}

// interior of a full-extent LayoutLeft field, C order [nx2][nx1][nx0]
std::vector<double> interior(const double* a, const int n[3], const int nx[3], const int ng3[3])
{
    std::vector<double> out((size_t)nx[0] * nx[1] * nx[2]);
    size_t o = 0;
    for (int k = 0; k < nx[2]; ++k) {
        for (int j = 0; j < nx[1]; ++j) {
            const size_t base = (size_t)ng3[0] + (size_t)n[0] * ((size_t)(j + ng3[1]) + (size_t)n[1] * (k + ng3[2]));
            for (int i = 0; i < nx[0]; ++i) {
                out[o++] = a[base + i];
            }
        }
    }
    return out;
}

void scatter_interior(const std::vector<double>& v, double* a, const int n[3], const int nx[3], const int ng3[3])
{
    size_t o = 0;
    for (int k = 0; k < nx[2]; ++k) {
        for (int j = 0; j < nx[1]; ++j) {
            const size_t base = (size_t)ng3[0] + (size_t)n[0] * ((size_t)(j + ng3[1]) + (size_t)n[1] * (k + ng3[2]));
            for (int i = 0; i < nx[0]; ++i) {
                a[base + i] = v[o++];
            }
        }
    }
}

bool write_container(const std::string& path, std::vector<Dataset>& sets)
{
    // index with provisional offsets, then fix the offsets once its length is known
    auto index_text = [&]() {
        std::ostringstream os;
        for (const Dataset& s : sets) {
            os << s.name << ' ' << (s.f64 ? "f64" : "i32") << ' ' << s.offset << ' ' << s.ext.size();
            for (int64_t e : s.ext) {
                os << ' ' << e;
            }
            os << '\n';
        }
        return os.str();
    };
    std::string idx;
    for (int pass = 0; pass < 3; ++pass) {
        idx = index_text();
        uint64_t off = 16 + idx.size();
        for (Dataset& s : sets) {
            off = (off + 63) / 64 * 64;
            s.offset = off;
            off += s.bytes();
        }
    }
    idx = index_text();
    std::ofstream f(path, std::ios::binary | std::ios::trunc);
    if (!f) {
        return false;
    }
    f.write(kMagic, 8);
    const uint64_t len = idx.size();
    f.write(reinterpret_cast<const char*>(&len), 8);
    f.write(idx.data(), (std::streamsize)idx.size());
    uint64_t pos = 16 + idx.size();
    static const char zeros[64] = {};
    for (const Dataset& s : sets) {
        f.write(zeros, (std::streamsize)(s.offset - pos));
        if (s.f64) {
            f.write(reinterpret_cast<const char*>(s.d.data()), (std::streamsize)s.bytes());
        } else {
            f.write(reinterpret_cast<const char*>(s.i.data()), (std::streamsize)s.bytes());
        }
        pos = s.offset + s.bytes();
    }
    return (bool)f;
}

bool read_container(const std::string& path, std::map<std::string, Dataset>& out)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) {
        return false;
    }
    char magic[8];
    uint64_t len = 0;
    f.read(magic, 8);
    f.read(reinterpret_cast<char*>(&len), 8);
    if (!f || std::memcmp(magic, kMagic, 8) != 0 || len > (1u << 24)) {
        return false;
    }
    std::string idx(len, '\0');
    f.read(idx.data(), (std::streamsize)len);
    std::istringstream is(idx);
    std::string line;
    while (std::getline(is, line)) {
        std::istringstream ls(line);
        Dataset s;
        std::string type;
        size_t rank = 0;
        ls >> s.name >> type >> s.offset >> rank;
        s.f64 = type == "f64";
        size_t count = 1;
        for (size_t r = 0; r < rank; ++r) {
            int64_t e = 0;
            ls >> e;
            s.ext.push_back(e);
            count *= (size_t)e;
        }
        if (!ls || (type != "f64" && type != "i32")) {
            return false;
        }
        f.seekg((std::streamoff)s.offset);
        if (s.f64) {
            s.d.resize(count);
            f.read(reinterpret_cast<char*>(s.d.data()), (std::streamsize)(count * 8));
        } else {
            s.i.resize(count);
            f.read(reinterpret_cast<char*>(s.i.data()), (std::streamsize)(count * 4));
        }
        if (!f) {
            return false;
        }
        out[s.name] = std::move(s);
    }
    return true;
}

// outputs written so far per (directory, prefix), for the XDMF time series
std::mutex g_series_mutex;
std::map<std::string, std::map<int, double>> g_series;

void write_xdmf(const std::string& dir, const std::string& prefix, const std::map<int, double>& outs,
                const std::vector<Dataset>& sets, int ndim, const int nx[3])
{
    std::ofstream x(dir + "/" + prefix + ".xmf", std::ios::trunc);
    if (!x) {
        return;
    }
    const int64_t nodes[3] = {nx[0] + 1, nx[1] + 1, nx[2] + 1};
    x << "<?xml version=\"1.0\" ?>\n<!DOCTYPE Xdmf SYSTEM \"Xdmf.dtd\" []>\n<Xdmf Version=\"3.0\">\n <Domain>\n"
      << "  <Grid Name=\"TimeSeries\" GridType=\"Collection\" CollectionType=\"Temporal\">\n";
    for (const auto& [id, t] : outs) {
        const std::string fn = file_name(prefix, id);
        auto item = [&](const Dataset& s, const std::string& dims) {
            std::ostringstream o;
            o << "<DataItem Format=\"Binary\" Endian=\"Little\" NumberType=\"Float\" Precision=\"8\" Seek=\""
              << s.offset << "\" Dimensions=\"" << dims << "\">" << fn << "</DataItem>";
            return o.str();
        };
        x << "   <Grid Name=\"output_" << id << "\" GridType=\"Uniform\">\n"
          << "    <Time Value=\"" << std::to_string(t) << "\"/>\n"
          << "    <Topology TopologyType=\"3DRectMesh\" Dimensions=\"" << nodes[2] << ' ' << nodes[1] << ' '
          << nodes[0] << "\"/>\n    <Geometry GeometryType=\"VXVYVZ\">\n";
        for (int d = 0; d < 3; ++d) {
            for (const Dataset& s : sets) {
                if (s.name == "x" + std::to_string(d) + "_ng") {
                    x << "     " << item(s, std::to_string(nodes[d])) << "\n";
                }
            }
        }
        x << "    </Geometry>\n";
        const std::string cdims =
            std::to_string(nx[2]) + " " + std::to_string(nx[1]) + " " + std::to_string(nx[0]);
        for (const Dataset& s : sets) {
            if (s.ext.size() == 3) {
                x << "    <Attribute Name=\"" << s.name << "\" AttributeType=\"Scalar\" Center=\"Cell\">\n     "
                  << item(s, cdims) << "\n    </Attribute>\n";
            }
        }
        x << "   </Grid>\n";
    }
    x << "  </Grid>\n </Domain>\n</Xdmf>\n";
    (void)ndim;
}

} // namespace

extern "C" {

int hcl_write_output(hcl_handle* h, const char* directory, const char* prefix, int output_id, int iter_output_id,
                     int time_output_id, int iter, double t)
{
    if (!h || !directory || !prefix) {
        return set_error(HCL_ERR_ARGUMENT, "null argument");
    }
    hcl_config cfg;
    int rc = hcl_get_config(h, &cfg);
    int n[3], nx[3], ng = 0;
    int64_t N = 0;
    if (rc || (rc = hcl_get_extents(h, n, &N)) || (rc = hcl_get_interior(h, nx, &ng))) {
        return rc;
    }
    const int nd = cfg.ndim, nfx = cfg.nfx;
    std::vector<double> rho((size_t)N), u((size_t)N * nd), P((size_t)N), T((size_t)N), fx((size_t)N * nfx);
    std::vector<double> rhou((size_t)N * nd), E((size_t)N);
    if ((rc = hcl_get_prim(h, rho.data(), u.data(), P.data(), T.data(), nfx > 0 ? fx.data() : nullptr, HCL_HOST)) ||
        (rc = hcl_get_state(h, rho.data(), rhou.data(), E.data(), nullptr, HCL_HOST))) {
        return rc;
    }
    std::vector<double> x[3];
    double* xp[3];
    for (int d = 0; d < 3; ++d) {
        x[d].resize((size_t)n[d] + 1);
        xp[d] = x[d].data();
    }
    if ((rc = hcl_get_grid(h, xp, nullptr, nullptr, nullptr, nullptr))) {
        return rc;
    }
    const int ng3[3] = {ng, nd > 1 ? ng : 0, nd > 2 ? ng : 0};
    std::vector<Dataset> sets;
    auto iscalar = [&](const char* name, int v) {
        Dataset s;
        s.name = name;
        s.f64 = false;
        s.i = {v};
        sets.push_back(std::move(s));
    };
    auto dscalar = [&](const char* name, double v) {
        Dataset s;
        s.name = name;
        s.d = {v};
        sets.push_back(std::move(s));
    };
    iscalar("output_id", output_id);
    iscalar("iter_output_id", iter_output_id);
    iscalar("time_output_id", time_output_id);
    iscalar("iter", iter);
    dscalar("current_time", t);
    dscalar("gamma", cfg.gamma);
    for (int d = 0; d < 3; ++d) {
        Dataset s;
        s.name = "x" + std::to_string(d);
        s.d = x[d];
        s.ext = {(int64_t)x[d].size()};
        sets.push_back(s);
        Dataset sn;
        sn.name = "x" + std::to_string(d) + "_ng";
        sn.d.assign(x[d].begin() + ng3[d], x[d].begin() + ng3[d] + nx[d] + 1);
        sn.ext = {(int64_t)nx[d] + 1};
        sets.push_back(std::move(sn));
    }
    auto field = [&](const std::string& name, const double* a) {
        Dataset s;
        s.name = name;
        s.d = interior(a, n, nx, ng3);
        s.ext = {nx[2], nx[1], nx[0]};
        sets.push_back(std::move(s));
    };
    field("rho", rho.data());
    for (int d = 0; d < nd; ++d) {
        field("ux" + std::to_string(d), u.data() + (size_t)N * d);
    }
    field("P", P.data());
    field("E", E.data());
    field("T", T.data());
    for (int f = 0; f < nfx; ++f) {
        field("fx" + std::to_string(f), fx.data() + (size_t)N * f);
    }
    const std::string dir(directory), pre(prefix);
    if (!write_container(dir + "/" + file_name(pre, output_id), sets)) {
        return set_error(HCL_ERR_ARGUMENT, "cannot write " + dir + "/" + file_name(pre, output_id));
    }
    std::lock_guard<std::mutex> lock(g_series_mutex);
    auto& outs = g_series[dir + "/" + pre];
    outs[output_id] = t;
    write_xdmf(dir, pre, outs, sets, nd, nx);
    return HCL_OK;
}

int hcl_read_restart(hcl_handle* h, const char* path, int* output_id, int* iter_output_id, int* time_output_id,
                     int* iter, double* t)
{
    if (!h || !path) {
        return set_error(HCL_ERR_ARGUMENT, "null argument");
    }
    std::map<std::string, Dataset> in;
    if (!read_container(path, in)) {
        return set_error(HCL_ERR_ARGUMENT, std::string("cannot read an output file at ") + path);
    }
    hcl_config cfg;
    int rc = hcl_get_config(h, &cfg);
    int n[3], nx[3], ng = 0;
    int64_t N = 0;
    if (rc || (rc = hcl_get_extents(h, n, &N)) || (rc = hcl_get_interior(h, nx, &ng))) {
        return rc;
    }
    const int nd = cfg.ndim, nfx = cfg.nfx;
    const int ng3[3] = {ng, nd > 1 ? ng : 0, nd > 2 ? ng : 0};
    // the file's grid must be the handle's (read_pdi checks the node counts,
    // io.cpp:356-358; here the nodes themselves)
    std::vector<double> x[3];
    double* xp[3];
    for (int d = 0; d < 3; ++d) {
        x[d].resize((size_t)n[d] + 1);
        xp[d] = x[d].data();
    }
    if ((rc = hcl_get_grid(h, xp, nullptr, nullptr, nullptr, nullptr))) {
        return rc;
    }
    for (int d = 0; d < 3; ++d) {
        const auto it = in.find("x" + std::to_string(d));
        if (it == in.end() || it->second.d != x[d]) {
            return set_error(HCL_ERR_CONFIG, "the output's x" + std::to_string(d) + " nodes differ from the handle's grid");
        }
    }
    const size_t cells = (size_t)nx[0] * nx[1] * nx[2];
    auto need = [&](const std::string& name) -> const Dataset* {
        const auto it = in.find(name);
        if (it == in.end() || !it->second.f64 || it->second.d.size() != cells) {
            return nullptr;
        }
        return &it->second;
    };
    std::vector<double> rho((size_t)N, 0.0), u((size_t)N * nd, 0.0), P((size_t)N, 0.0), fx((size_t)N * nfx, 0.0);
    const Dataset* r = need("rho");
    const Dataset* p = need("P");
    if (!r || !p) {
        return set_error(HCL_ERR_CONFIG, "the output lacks rho or P of this grid's size");
    }
    scatter_interior(r->d, rho.data(), n, nx, ng3);
    scatter_interior(p->d, P.data(), n, nx, ng3);
    for (int d = 0; d < nd; ++d) {
        const Dataset* s = need("ux" + std::to_string(d));
        if (!s) {
            return set_error(HCL_ERR_CONFIG, "the output lacks ux" + std::to_string(d));
        }
        scatter_interior(s->d, u.data() + (size_t)N * d, n, nx, ng3);
    }
    for (int f = 0; f < nfx; ++f) {
        const Dataset* s = need("fx" + std::to_string(f));
        if (!s) {
            return set_error(HCL_ERR_CONFIG, "the output lacks fx" + std::to_string(f));
        }
        scatter_interior(s->d, fx.data() + (size_t)N * f, n, nx, ng3);
    }
    auto ival = [&](const char* name, int* dst) {
        const auto it = in.find(name);
        if (dst && it != in.end() && !it->second.f64 && it->second.i.size() == 1) {
            *dst = it->second.i[0];
        }
    };
    int it_file = 0;
    double t_file = 0.0;
    ival("output_id", output_id);
    ival("iter_output_id", iter_output_id);
    ival("time_output_id", time_output_id);
    ival("iter", &it_file);
    const auto tt = in.find("current_time");
    if (tt == in.end() || tt->second.d.size() != 1) {
        return set_error(HCL_ERR_CONFIG, "the output lacks current_time");
    }
    t_file = tt->second.d[0];
    if ((rc = hcl_set_state_from_prim(h, rho.data(), u.data(), P.data(), nfx > 0 ? fx.data() : nullptr)) ||
        (rc = hcl_set_clock(h, t_file, it_file))) {
        return rc;
    }
    if (iter) {
        *iter = it_file;
    }
    if (t) {
        *t = t_file;
    }
    return HCL_OK;
}

} // extern "C"
