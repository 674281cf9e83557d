// Output files in the reference's formats (src/io.h, src/solver.h), so that
// its readers (script/read_bin.py, the reconstructor) consume them.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace dalm {

struct OutVar {
    std::string name;
    int64_t dim;          // components per cell (AoS)
    const double *data;   // [cells][dim], reference layout over the stored grid
};

// Header::write + write_binary (src/io.h:34-45, 303-320): int64 size[3],
// gc, var count, var dims, (length, name) per var; then x, y, z and every
// variable's array, all native-endian.
void write_field_binary(const std::string &path, const int64_t size[3], int64_t gc,
                        const std::vector<double> &x, const std::vector<double> &y,
                        const std::vector<double> &z, const std::vector<OutVar> &vars);

// make_rank_binary_filename (src/io.h:322-324): prefix_RRRRR_SSSSSSSSSS
std::string binary_filename(const std::string &prefix, int rank, int64_t step);

// A JSON number: the shortest decimal that reads back as v, with ".0"
// appended to integral values, as the reference's JSON library prints it.
std::string json_number(double v);

struct SnapshotEntry {
    int64_t step;
    double time;
    bool tavg;
};
// snapshot.json (src/solver.h:1234-1253): [{"step", ["tavg": "yes",] "time"}]
void write_snapshot_json(const std::string &path, const std::vector<SnapshotEntry> &entries);
// partition.json of one rank holding the whole grid (src/solver.h:980-998)
void write_partition_json(const std::string &path, const int64_t size[3], int64_t gc);

// ap_info.log (src/solver.h:949-974): the blade-point tables after set-up,
// per point r, dr, chord, twist and its Cd / Cl columns over the
// angle-of-attack list ([ap][atk] row-major), then that list; "%lf" numbers.
void write_ap_info(const std::string &path, int64_t ap_count, int64_t atk_count,
                   const std::vector<double> &r, const std::vector<double> &dr,
                   const std::vector<double> &chord, const std::vector<double> &twist,
                   const std::vector<double> &cd, const std::vector<double> &cl,
                   const std::vector<double> &atk);

}  // namespace dalm
