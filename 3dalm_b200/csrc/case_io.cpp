#include "case_io.hpp"

#include <cmath>
#include <fstream>
#include <sstream>
#include <stdexcept>

#include "json_lite.hpp"

namespace dalm {

namespace {

constexpr double PI_D = 3.14159265358979323846;

Json read_json(const std::string &path) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("cannot open " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    try {
        return Json::parse(ss.str());
    } catch (const std::exception &e) {
        throw std::runtime_error(path + ": " + e.what());
    }
}

// dx[i] = (x[i+1]-x[i-1])/2 with one-sided ends (src/io.h:112-125)
std::vector<double> spacing(const std::vector<double> &c) {
    size_t n = c.size();
    std::vector<double> d(n);
    for (size_t i = 1; i + 1 < n; i++) d[i] = 0.5 * (c[i + 1] - c[i - 1]);
    d[0] = -1.5 * c[0] + 2.0 * c[1] - 0.5 * c[2];
    d[n - 1] = 1.5 * c[n - 1] - 2.0 * c[n - 2] + 0.5 * c[n - 3];
    return d;
}

// find_floor_index (src/util.h:119-146)
int64_t floor_index(const std::vector<double> &a, double v) {
    int64_t n = (int64_t)a.size();
    if (v < a[0]) return -1;
    if (v >= a[n - 1]) return n - 1;
    int64_t lo = 0, hi = n - 1, found = -1;
    while (lo <= hi) {
        int64_t mid = lo + (hi - lo) / 2;
        if (a[mid] <= v) {
            found = mid;
            lo = mid + 1;
        } else {
            hi = mid - 1;
        }
    }
    return found;
}

// build_A scaling factor: max over interior cells of |a_c| (src/eq.h:716-778)
double max_diagonal(const CaseData &c) {
    double md = 0;
    int64_t gc = c.gc, NX = c.size[0], NY = c.size[1], NZ = c.size[2];
    std::vector<double> ax(NX, 0.0), ay(NY, 0.0), az(NZ, 0.0);
    // per-axis parts in the reference's subtraction order; the diagonal is
    // (((((0 - ex) - aw) - an) - as) - at) - ab, assembled below per cell
    for (int64_t i = gc; i < NX - gc; i++) {
        double acx = 0;
        if (i < NX - gc - 1) acx -= 1 / (c.dx[i] * (c.x[i + 1] - c.x[i]));
        else acx -= 2 / (c.dx[i] * c.dx[i]);
        ax[i] = acx;
    }
    for (int64_t i = gc; i < NX - gc; i++) {
        double ex = -ax[i];
        double aw = i > gc ? 1 / (c.dx[i] * (c.x[i] - c.x[i - 1])) : 0.0;
        for (int64_t j = gc; j < NY - gc; j++) {
            double an = j < NY - gc - 1 ? 1 / (c.dy[j] * (c.y[j + 1] - c.y[j])) : 0.0;
            double as = j > gc ? 1 / (c.dy[j] * (c.y[j] - c.y[j - 1])) : 0.0;
            double pre = ((0.0 - ex) - aw) - an;
            pre = pre - as;
            for (int64_t k = gc; k < NZ - gc; k++) {
                double at = k < NZ - gc - 1 ? 1 / (c.dz[k] * (c.z[k + 1] - c.z[k])) : 0.0;
                double ab = k > gc ? 1 / (c.dz[k] * (c.z[k] - c.z[k - 1])) : 0.0;
                double ac = (pre - at) - ab;
                if (std::fabs(ac) > md) md = std::fabs(ac);
            }
        }
    }
    return md;
}

}  // namespace

CaseData load_case(const std::string &dir) {
    CaseData c;
    c.dir = dir;
    Json setup = read_json(dir + "/setup.json");
    Json mesh = read_json(dir + "/mesh.json");

    // mesh (src/io.h:98-164)
    c.gc = (int64_t)mesh["guide cell"].number();
    c.x = mesh["x"].numbers();
    c.y = mesh["y"].numbers();
    c.z = mesh["z"].numbers();
    c.size[0] = (int64_t)c.x.size();
    c.size[1] = (int64_t)c.y.size();
    c.size[2] = (int64_t)c.z.size();
    if (c.gc < 2) throw std::runtime_error("mesh.json: guide cell must be >= 2 (src/solver.h:615)");
    for (int a = 0; a < 3; a++)
        if (c.size[a] < 2 * c.gc + 2)
            throw std::runtime_error("mesh.json: too few cells along an axis");
    const std::vector<double> *axes[3] = {&c.x, &c.y, &c.z};
    for (int a = 0; a < 3; a++)
        for (size_t i = 1; i < axes[a]->size(); i++)
            if (!((*axes[a])[i] > (*axes[a])[i - 1]))
                throw std::runtime_error("mesh.json: cell centres must increase strictly");
    c.dx = spacing(c.x);
    c.dy = spacing(c.y);
    c.dz = spacing(c.z);

    // runtime / output (src/solver.h:589-597, src/solver.h:193-199)
    c.dt = setup["runtime"]["dt"].number();
    double total_time = setup["runtime"]["time"].number();
    c.max_step = (int64_t)(total_time / c.dt);
    c.tavg_start_time = setup["output"]["time avg start time"].number();
    c.output_start_time = setup["output"]["output start time"].number();
    c.output_interval_time = setup["output"]["output interval time"].number();
    if (setup.contains("turbulence grid")) {  // src/solver.h:599-611
        const Json &tg = setup["turbulence grid"];
        c.has_grid = true;
        c.grid_thick = tg["thick"].number();
        c.grid_mesh = tg["mesh"].number();
        c.grid_bar = tg["bar"].number();
        for (int m = 0; m < 3; m++) c.grid_at[m] = tg["placement"][m].number();
    }
    if (setup.contains("floor start")) {  // src/solver.h:618-625
        c.retracted_floor = true;
        c.floor_start = setup["floor start"].number();
    }
    if (setup.contains("probe")) {  // src/solver.h:656-664
        const Json &pr = setup["probe"];
        for (size_t m = 0; m < pr.size(); m++)
            for (int a = 0; a < 3; a++) c.probes.push_back(pr[m][a].number());
    }

    // inflow / cfd (src/solver.h:627-635)
    for (int m = 0; m < 3; m++) c.uin[m] = setup["inflow"]["value"][m].number();
    c.re = setup["cfd"]["Re"].number();
    c.cs = setup["cfd"]["Cs"].number();

    // eq (src/solver.h:639-652)
    const Json &eq = setup["eq"];
    c.tol = eq["tolerance"].number();
    c.max_it = (int64_t)eq["max iteration"].number();
    c.method = eq["method"].string();
    if (c.method == "BiCG") {
        const Json &pc = eq["preconditioner"];
        c.pc_method = pc["method"].string();
        c.pc_max_it = (int64_t)pc["max iteration"].number();
        if (c.pc_method == "SOR") c.pc_relax = pc["relaxation rate"].number();
        else if (c.pc_method != "Jacobi")
            throw std::runtime_error("setup.json: preconditioner method must be \"Jacobi\" or \"SOR\"");
    } else if (c.method == "SOR") {
        c.relax = eq["relaxation rate"].number();
    } else if (c.method != "Jacobi") {
        throw std::runtime_error("setup.json: eq method must be \"SOR\", \"BiCG\" or \"Jacobi\"");
    }

    // turbines (src/solver.h:702-708, src/alm.h:144-206, 35-142)
    if (setup.contains("windturbine array")) {
        const Json &arr = setup["windturbine array"];
        const Json &alm = setup["alm"];
        c.ap_per_blade = (int64_t)alm["blade points"].number();
        c.projection_width = alm["projection width"].number();
        Json wtp = read_json(dir + "/windturbine.json");
        c.blades = (int64_t)wtp["number of blades"].number();
        double tower = wtp["tower"].number(), overhang = wtp["overhang"].number();
        for (size_t w = 0; w < arr.size(); w++) {
            const Json &tj = arr[w];
            TurbineSpec t;
            for (int m = 0; m < 3; m++) t.base[m] = tj["base"][m].number();
            t.rot_speed = tj["rotation speed"].number();
            t.rot_center[0] = -overhang;
            t.rot_center[1] = 0;
            t.rot_center[2] = tower;
            // First non-zero or object slot wins (src/alm.h:167-204).  All-zero
            // slots leave the reference's angle type indeterminate; here they
            // mean no rotation.
            t.angle_type = 3;
            t.formula[0] = t.formula[1] = t.formula[2] = t.formula[3] = 0;
            const Json &ang = tj["angle"];
            for (int s = 0; s < 3 && s < (int)ang.size(); s++) {
                const Json &a = ang[s];
                if ((a.is_number() && a.number() != 0) || a.is_object()) {
                    t.angle_type = s;  // roll, pitch, yaw
                    if (a.is_number()) {
                        t.formula[3] = a.number() * PI_D / 180;
                    } else {
                        t.formula[0] = a["amp"].number() * PI_D / 180;
                        t.formula[1] = 2 * PI_D / a["T"].number();
                        t.formula[2] = a["phase"].number() * PI_D / 180;
                        t.formula[3] = a["offset"].number() * PI_D / 180;
                    }
                    break;
                }
            }
            c.turbines.push_back(t);
        }
        // blade points (src/alm.h:35-103)
        const Json &blade = wtp["blade"];
        const Json &foils = blade["airfoil"];
        c.atk = blade["attack angle"].numbers();
        c.atk_count = (int64_t)c.atk.size();
        std::vector<double> afr, aftw, afch;
        std::vector<std::vector<double>> afcd, afcl;
        for (size_t s = 0; s < foils.size(); s++) {
            afr.push_back(foils[s]["r/R"].number());
            aftw.push_back(foils[s]["twist[deg]"].number());
            afch.push_back(foils[s]["chord/R"].number());
            afcd.push_back(foils[s]["Cd"].numbers());
            afcl.push_back(foils[s]["Cl"].numbers());
            if ((int64_t)afcd.back().size() != c.atk_count || (int64_t)afcl.back().size() != c.atk_count)
                throw std::runtime_error("windturbine.json: Cd/Cl length differs from the attack-angle table");
        }
        int64_t S = (int64_t)afr.size();
        int64_t ap_per_wt = c.blades * c.ap_per_blade;
        int64_t ap_count = (int64_t)c.turbines.size() * ap_per_wt;
        double wt_r = wtp["R"].number(), hub_r = wtp["hub R"].number();
        double dr = (wt_r - hub_r) / c.ap_per_blade;
        c.ap_cd.assign(ap_count * c.atk_count, 0.0);
        c.ap_cl.assign(ap_count * c.atk_count, 0.0);
        for (int64_t a = 0; a < ap_count; a++) {
            double r = hub_r + (a % c.ap_per_blade + 0.5) * dr;
            c.ap_r.push_back(r);
            c.ap_dr.push_back(dr);
            int64_t af = floor_index(afr, r);
            double *cd = &c.ap_cd[a * c.atk_count], *cl = &c.ap_cl[a * c.atk_count];
            if (af < 0 || af >= S - 1) {
                int64_t s = af < 0 ? 0 : S - 1;
                c.ap_chord.push_back(afch[s]);
                c.ap_twist.push_back(aftw[s]);
                for (int64_t j = 0; j < c.atk_count; j++) {
                    cd[j] = afcd[s][j];
                    cl[j] = afcl[s][j];
                }
            } else {
                double a1 = (r - afr[af]) / (afr[af + 1] - afr[af]);
                double a0 = 1 - a1;
                c.ap_chord.push_back(a0 * afch[af] + a1 * afch[af + 1]);
                c.ap_twist.push_back(a0 * aftw[af] + a1 * aftw[af + 1]);
                for (int64_t j = 0; j < c.atk_count; j++) {
                    cd[j] = a0 * afcd[af][j] + a1 * afcd[af + 1][j];
                    cl[j] = a0 * afcl[af][j] + a1 * afcl[af + 1][j];
                }
            }
        }
    }
    c.max_diag = max_diagonal(c);
    return c;
}

}  // namespace dalm
