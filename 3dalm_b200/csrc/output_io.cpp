#include "output_io.hpp"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace dalm {

namespace {

std::ofstream open_out(const std::string &path, bool binary) {
    std::ofstream f(path, binary ? std::ios::binary : std::ios::out);
    if (!f) throw std::runtime_error("cannot write " + path);
    return f;
}

void put_i64(std::ofstream &f, int64_t v) { f.write((const char *)&v, sizeof v); }

std::string int_array(const int64_t v[3], const std::string &indent) {
    std::ostringstream o;
    o << "[\n";
    for (int m = 0; m < 3; m++) o << indent << "  " << v[m] << (m < 2 ? ",\n" : "\n");
    o << indent << "]";
    return o.str();
}

}  // namespace

void write_field_binary(const std::string &path, const int64_t size[3], int64_t gc,
                        const std::vector<double> &x, const std::vector<double> &y,
                        const std::vector<double> &z, const std::vector<OutVar> &vars) {
    std::ofstream f = open_out(path, true);
    for (int m = 0; m < 3; m++) put_i64(f, size[m]);
    put_i64(f, gc);
    put_i64(f, (int64_t)vars.size());
    for (const OutVar &v : vars) put_i64(f, v.dim);
    for (const OutVar &v : vars) {
        put_i64(f, (int64_t)v.name.size());
        f.write(v.name.data(), (std::streamsize)v.name.size());
    }
    f.write((const char *)x.data(), (std::streamsize)(size[0] * sizeof(double)));
    f.write((const char *)y.data(), (std::streamsize)(size[1] * sizeof(double)));
    f.write((const char *)z.data(), (std::streamsize)(size[2] * sizeof(double)));
    const int64_t cells = size[0] * size[1] * size[2];
    for (const OutVar &v : vars)
        f.write((const char *)v.data, (std::streamsize)(cells * v.dim * sizeof(double)));
    if (!f) throw std::runtime_error("write failed: " + path);
}

std::string binary_filename(const std::string &prefix, int rank, int64_t step) {
    char buf[64];
    std::snprintf(buf, sizeof buf, "_%05d_%010lld", rank, (long long)step);
    return prefix + buf;
}

std::string json_number(double v) {
    char buf[40];
    for (int p = 1; p <= 17; p++) {
        std::snprintf(buf, sizeof buf, "%.*g", p, v);
        if (std::strtod(buf, nullptr) == v) break;
    }
    std::string s(buf);
    if (s.find_first_of(".eEn") == std::string::npos) s += ".0";
    return s;
}

void write_snapshot_json(const std::string &path, const std::vector<SnapshotEntry> &entries) {
    std::ofstream f = open_out(path, false);
    f << "[";
    for (size_t n = 0; n < entries.size(); n++) {
        const SnapshotEntry &e = entries[n];
        f << (n ? ",\n" : "\n") << "  {\n    \"step\": " << e.step << ",\n";
        if (e.tavg) f << "    \"tavg\": \"yes\",\n";
        f << "    \"time\": " << json_number(e.time) << "\n  }";
    }
    f << (entries.empty() ? "]" : "\n]");
}

void write_partition_json(const std::string &path, const int64_t size[3], int64_t gc) {
    const int64_t zero[3] = {0, 0, 0};
    std::ofstream f = open_out(path, false);
    f << "{\n  \"gc\": " << gc << ",\n  \"partition\": [\n    {\n      \"offset\": "
      << int_array(zero, "      ") << ",\n      \"rank\": 0,\n      \"size\": "
      << int_array(size, "      ") << "\n    }\n  ],\n  \"size\": " << int_array(size, "  ")
      << "\n}";
}

void write_ap_info(const std::string &path, int64_t ap_count, int64_t atk_count,
                   const std::vector<double> &r, const std::vector<double> &dr,
                   const std::vector<double> &chord, const std::vector<double> &twist,
                   const std::vector<double> &cd, const std::vector<double> &cl,
                   const std::vector<double> &atk) {
    FILE *f = std::fopen(path.c_str(), "w");
    if (!f) throw std::runtime_error("cannot write " + path);
    std::fprintf(f, "ap count = %ld, atk acount = %ld\n", (long)ap_count, (long)atk_count);
    for (int64_t a = 0; a < ap_count; a++) {
        std::fprintf(f, "ap %ld\n", (long)a);
        std::fprintf(f, "\tr = %lf\n", r[a]);
        std::fprintf(f, "\tdr = %lf\n", dr[a]);
        std::fprintf(f, "\tchord = %lf\n", chord[a]);
        std::fprintf(f, "\ttwist = %lf\n", twist[a]);
        std::fprintf(f, "\tcd = \n");
        for (int64_t j = 0; j < atk_count; j++) std::fprintf(f, "\t\t%lf\n", cd[a * atk_count + j]);
        std::fprintf(f, "\tcl = \n");
        for (int64_t j = 0; j < atk_count; j++) std::fprintf(f, "\t\t%lf\n", cl[a * atk_count + j]);
    }
    std::fprintf(f, "atk\n");
    for (int64_t j = 0; j < atk_count; j++) std::fprintf(f, "\t%lf\n", atk[j]);
    std::fclose(f);
}

}  // namespace dalm
