// Case loading: setup.json, mesh.json, windturbine.json with the semantics
// of Solver::initialize (src/solver.h:564-708), build_mesh_from_json
// (src/io.h:98-164), build_wt_props / build_ap_props (src/alm.h:35-206) and
// build_A's scaling factor (src/eq.h:701-798).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace dalm {

struct TurbineSpec {
    double base[3];
    double rot_center[3];
    int angle_type;     // EulerAngleType
    double formula[4];  // angle = f0 sin(f1 t + f2) + f3
    double rot_speed;
};

struct CaseData {
    std::string dir;
    int64_t size[3] = {0, 0, 0};
    int64_t gc = 0;
    std::vector<double> x, y, z, dx, dy, dz;
    double uin[3] = {0, 0, 0};
    double re = 0, cs = 0, dt = 0;
    int64_t max_step = 0;
    double tavg_start_time = 0;
    double output_start_time = 0, output_interval_time = 0;
    std::string method, pc_method;  // "SOR" | "BiCG" | "Jacobi"; "Jacobi" | "SOR"
    int64_t max_it = 0, pc_max_it = 0;
    double tol = 0, relax = 1, pc_relax = 1;
    double max_diag = 0;
    // turbulence-generating grid (src/solver.h:599-611): bar width, mesh
    // spacing, thickness, placement
    bool has_grid = false;
    double grid_bar = 0, grid_mesh = 0, grid_thick = 0, grid_at[3] = {0, 0, 0};
    // retracted floor (src/solver.h:618-625): slip z- wall for x < floor_start
    bool retracted_floor = false;
    double floor_start = 0;
    // probes (src/solver.h:656-699): requested points
    std::vector<double> probes;  // [n][3]
    // actuator line
    int64_t blades = 0, ap_per_blade = 0, atk_count = 0;
    double projection_width = 0;
    std::vector<TurbineSpec> turbines;
    std::vector<double> ap_r, ap_dr, ap_chord, ap_twist;  // per point
    std::vector<double> ap_cd, ap_cl;                     // [ap][atk]
    std::vector<double> atk;
    int64_t ap_count() const { return (int64_t)ap_r.size(); }
};

// Throws std::runtime_error with a readable message on any problem.
CaseData load_case(const std::string &dir);

}  // namespace dalm
