// Command-line driver:
//   dalm <case_dir> [--steps N] [--quiet] [--no-output] [--reference-sums] [--mixed]
//        [--fused-jacobi]
// Mirrors the reference's `solver <case_dir>` (src/solver.cpp:6-47): runs
// steps 0..max_step (or N steps), prints the per-step line
// `step time it err avg_div max_cfl` (src/solver.h:1188-1190), writes the
// reference's output files into <case_dir>/output (unless --no-output), then
// prints the per-turbine thrust, torque and power.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <vector>

#include <string>

#include "../../include/dalm.h"

// Reads exactly v.size() doubles; false when the file is absent.
static bool read_raw(const std::string &path, std::vector<double> &v) {
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) return false;
    size_t n = fread(v.data(), sizeof(double), v.size(), f);
    fclose(f);
    if (n != v.size()) {
        fprintf(stderr, "%s: expected %zu doubles, read %zu\n", path.c_str(), v.size(), n);
        exit(1);
    }
    return true;
}

int main(int argc, char **argv) {
    if (argc < 2) {
        fprintf(stderr,
                "usage: %s <case_dir> [--steps N] [--quiet] [--no-output] [--reference-sums] "
                "[--mixed] [--fused-jacobi]\n",
                argv[0]);
        return 2;
    }
    const char *dir = argv[1];
    long long steps = -1;
    bool quiet = false;
    dalm_options opt;
    dalm_default_options(&opt);
    opt.write_output = 1;
    for (int a = 2; a < argc; a++) {
        if (!strcmp(argv[a], "--steps") && a + 1 < argc) steps = atoll(argv[++a]);
        else if (!strcmp(argv[a], "--quiet")) quiet = true;
        else if (!strcmp(argv[a], "--no-output")) opt.write_output = 0;
        else if (!strcmp(argv[a], "--reference-sums")) opt.reference_sums = 1;
        else if (!strcmp(argv[a], "--mixed")) opt.precision = DALM_MIXED;
        else if (!strcmp(argv[a], "--fused-jacobi")) opt.fused_jacobi = 1;
        else {
            fprintf(stderr, "unknown option %s\n", argv[a]);
            return 2;
        }
    }
    time_t t0 = time(0);
    printf("START %s\n", ctime(&t0));
    dalm_handle *h = nullptr;
    int rc = dalm_create(dir, &opt, &h);
    if (rc != DALM_OK) {
        fprintf(stderr, "dalm_create failed (%d): %s\n", rc, dalm_last_error(nullptr));
        return 1;
    }
    // Optional initial state written by the case generator (casegen.py):
    // inflow_profile.f64 ([NY][NZ][3]) and initial_U.f64 ([NX][NY][NZ][3]),
    // raw little-endian float64.  The reference always starts from uniform Uin.
    int64_t size[3], gc;
    dalm_get_size(h, size, &gc);
    size_t cells = (size_t)(size[0] * size[1] * size[2]);
    std::vector<double> prof((size_t)(size[1] * size[2] * 3)), U(cells * 3);
    if (read_raw(std::string(dir) + "/inflow_profile.f64", prof)) {
        if (dalm_set_inflow_profile(h, prof.data()) != DALM_OK) {
            fprintf(stderr, "dalm_set_inflow_profile: %s\n", dalm_last_error(h));
            return 1;
        }
    }
    if (read_raw(std::string(dir) + "/initial_U.f64", U)) {
        if (dalm_set_state(h, U.data(), nullptr, nullptr,
                           DALM_SET_APPLY_UBC | DALM_SET_RECOMPUTE_JU) != DALM_OK) {
            fprintf(stderr, "dalm_set_state: %s\n", dalm_last_error(h));
            return 1;
        }
    }
    U.clear();
    U.shrink_to_fit();
    double dt = 0;
    int64_t max_step = 0;
    dalm_get_runtime(h, &dt, &max_step);
    long long total = steps >= 0 ? steps : (long long)max_step + 1;
    for (long long s = 0; s < total; s++) {
        rc = dalm_step(h, 1);
        if (rc != DALM_OK) {
            fprintf(stderr, "dalm_step failed (%d): %s\n", rc, dalm_last_error(h));
            dalm_destroy(h);
            return 1;
        }
        int64_t step = 0, it = 0;
        double err = 0, avg_div = 0, cfl = 0;
        dalm_get_step_stats(h, &step, &it, &err, &avg_div, &cfl);
        if (!quiet && step > 1)
            printf("%lld %e %lld %e %e %e\n", (long long)(step - 1), dt * (double)(step - 1),
                   (long long)it, err, avg_div, cfl);
    }
    int64_t counts[5];
    dalm_get_counts(h, counts);
    if (counts[0] > 0) {
        std::vector<double> th(counts[0]), tq(counts[0]), pw(counts[0]);
        dalm_get_turbines(h, th.data(), tq.data(), pw.data());
        for (int64_t w = 0; w < counts[0]; w++)
            printf("turbine %lld thrust %e torque %e power %e\n", (long long)w, th[w], tq[w], pw[w]);
    }
    dalm_destroy(h);
    time_t t1 = time(0);
    printf("END %s\n", ctime(&t1));
    return 0;
}
