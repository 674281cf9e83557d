/*
 * Multi-rank CPU run of the reference solver (BASELINE INFRASTRUCTURE ONLY:
 * the timed CPU baseline beside the GPU benchmark; never part of the
 * product).  Built by oracle/Makefile into oracle/_ref/ref_mpirun from the
 * reference's own sources where they lie, with the shared-memory MPI subset
 * in shm/mpi.h standing in for an MPI library, OpenACC off.
 *
 *   ref_mpirun <case_dir> --ranks N --warmup W --steps K --out result.json
 *              [--state initial_U.f64] [--profile inflow_profile.f64] [--budget S]
 *
 * The launcher maps one shared region, forks N ranks and waits for them.
 * Each rank is exactly what `mpirun -n N solver <case_dir>` would start:
 * Solver::initialize partitions the grid into x-slabs (calc_partition,
 * src/solver.h:27-50) and every stage exchanges halos and reduces through the
 * MPI calls.  The ranks then load their slab of the initial velocity (global
 * layout U[NX][NY][NZ][3], guide cells included), derive the state as
 * Solver::initialize does (src/solver.h:767-833, with the inflow profile
 * extension), run W untimed steps and K timed steps of src/solver.h:1034-1306
 * (stages in ref_stages.hpp).  Every step ends with a barrier; rank 0 times
 * each step with the monotonic clock.  With --budget S no timed step begins
 * once S seconds have passed since the start (every step that runs is
 * whole); steps_timed says how many ran.
 *
 * result.json: ranks, cells, warmup, steps, steps_timed, per-step seconds and
 * Poisson iterations / residuals of the timed steps (0 for step 0, which
 * solves nothing), and the set-up and warm-up seconds.  Exit status 0 on success; if any rank fails the others are
 * killed and the status is non-zero.
 */
#include "solver.h"
#include "ref_stages.hpp"

#include <cerrno>
#include <csignal>
#include <cstdio>
#include <string>
#include <vector>

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/wait.h>
#include <unistd.h>

using namespace refstages;

namespace {

constexpr int MAX_STEPS = 4096;

struct Result {
    int ok, steps_done;
    int64_t cells;
    double init_s, warmup_s;
    int64_t it[MAX_STEPS];
    double err[MAX_STEPS], secs[MAX_STEPS];
};

struct Args {
    std::string case_dir, out, state, profile;
    int ranks = 1, warmup = 0, steps = 1;
    double budget = 0;  // seconds since start after which no further timed step begins (0: none)
};

double now() { return shm_mpi::now_s(); }

bool read_at(int fd, void *dst, size_t bytes, off_t off) {
    char *p = (char *)dst;
    while (bytes > 0) {
        ssize_t n = pread(fd, p, bytes, off);
        if (n <= 0) return false;
        p += n;
        bytes -= (size_t)n;
        off += n;
    }
    return true;
}

int rank_main(const Args &a, Result *res) {
    double t0 = now();
    RefCase c;
    std::string prog = "solver", dir = a.case_dir;
    char *argv[] = {&prog[0], &dir[0], nullptr};
    c.solver.initialize(2, argv);
    Solver &s = c.solver;
    const Int NY = s.gsize[1], NZ = s.gsize[2];
    if (!a.profile.empty()) {
        int fd = open(a.profile.c_str(), O_RDONLY);
        c.profile.resize((size_t)NY * NZ * 3);
        if (fd < 0 || !read_at(fd, c.profile.data(), c.profile.size() * sizeof(Real), 0)) {
            std::fprintf(stderr, "cannot read %s\n", a.profile.c_str());
            return 2;
        }
        close(fd);
        c.has_profile = true;
    }
    if (!a.state.empty()) {
        // this rank's planes: local i <-> global i + offset[0]
        int fd = open(a.state.c_str(), O_RDONLY);
        const size_t plane = (size_t)NY * NZ * 3 * sizeof(Real);
        bool ok = fd >= 0;
        for (Int i = 0; ok && i < s.size[0]; i++)
            ok = read_at(fd, s.cfd.U[(size_t)i * NY * NZ], plane, (off_t)((i + s.offset[0]) * plane));
        if (fd >= 0) close(fd);
        if (!ok) {
            std::fprintf(stderr, "cannot read %s\n", a.state.c_str());
            return 2;
        }
    }
    derive_state(&c, 3);
    MPI_Barrier(MPI_COMM_WORLD);
    double t1 = now();
    for (int n = 0; n < a.warmup; n++) do_step(&c);
    MPI_Barrier(MPI_COMM_WORLD);
    double t2 = now();
    int done = 0;
    for (int n = 0; n < a.steps; n++) {
        const bool solves = s.rt.step != 0;  // step 0 integrates nothing (src/solver.h:1038)
        double ts = now();
        do_step(&c);
        MPI_Barrier(MPI_COMM_WORLD);
        done = n + 1;
        if (s.mpi.rank == 0) {
            res->secs[n] = now() - ts;
            res->it[n] = solves ? s.eq.it : 0;
            res->err[n] = solves ? s.eq.err : 0.0;
        }
        // the wall budget: rank 0's clock decides for every rank
        int stop = (s.mpi.rank == 0 && a.budget > 0 && now() - t0 > a.budget) ? 1 : 0;
        MPI_Allreduce(MPI_IN_PLACE, &stop, 1, MPI_INT, MPI_MAX, MPI_COMM_WORLD);
        if (stop) break;
    }
    if (s.mpi.rank == 0) {
        res->steps_done = done;
        res->cells = (s.gsize[0] - 2 * s.gc) * (s.gsize[1] - 2 * s.gc) * (s.gsize[2] - 2 * s.gc);
        res->init_s = t1 - t0;
        res->warmup_s = t2 - t1;
        res->ok = 1;
    }
    std::fflush(stdout);
    return 0;
}

bool parse(int argc, char **argv, Args &a) {
    if (argc < 2) return false;
    a.case_dir = argv[1];
    for (int i = 2; i + 1 < argc; i += 2) {
        std::string k = argv[i], v = argv[i + 1];
        if (k == "--ranks") a.ranks = std::stoi(v);
        else if (k == "--warmup") a.warmup = std::stoi(v);
        else if (k == "--steps") a.steps = std::stoi(v);
        else if (k == "--out") a.out = v;
        else if (k == "--state") a.state = v;
        else if (k == "--profile") a.profile = v;
        else if (k == "--budget") a.budget = std::stod(v);
        else return false;
    }
    return a.ranks >= 1 && a.ranks <= shm_mpi::MAX_RANKS && a.steps >= 1 && a.steps <= MAX_STEPS &&
           a.warmup >= 0 && !a.out.empty();
}

// Mailbox size: the largest halo message, 3 components x gc planes of the
// y-z cross-section (src/cfd.h:253-301), read from mesh.json's sizes.
size_t halo_bytes(const std::string &case_dir) {
    json m = json::parse(std::ifstream(case_dir + "/mesh.json"));
    size_t ny = m["y"].size(), nz = m["z"].size(), gc = m["guide cell"];
    return 3 * gc * ny * nz * sizeof(Real);
}

}  // namespace

int main(int argc, char **argv) {
    Args a;
    if (!parse(argc, argv, a)) {
        std::fprintf(stderr,
                     "usage: ref_mpirun <case_dir> --ranks N --warmup W --steps K --out file "
                     "[--state f] [--profile f]\n");
        return 2;
    }
    shm_mpi::World *w = shm_mpi::create(a.ranks, halo_bytes(a.case_dir));
    void *rp = mmap(nullptr, sizeof(Result), PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
    if (!w || rp == MAP_FAILED) {
        std::perror("mmap");
        return 3;
    }
    Result *res = (Result *)rp;
    std::memset(res, 0, sizeof(Result));
    std::fflush(stdout);
    std::vector<pid_t> pids;
    for (int r = 0; r < a.ranks; r++) {
        pid_t pid = fork();
        if (pid < 0) {
            std::perror("fork");
            for (pid_t p : pids) kill(p, SIGKILL);
            return 3;
        }
        if (pid == 0) {
            shm_mpi::join(w, r);
            int rc = rank_main(a, res);
            std::fflush(nullptr);
            _exit(rc);
        }
        pids.push_back(pid);
    }
    int failed = 0;
    for (size_t n = 0; n < pids.size(); n++) {
        int status = 0;
        pid_t p = wait(&status);
        if (p < 0) break;
        if (!WIFEXITED(status) || WEXITSTATUS(status) != 0) {
            if (!failed) std::fprintf(stderr, "ref_mpirun: rank process %d failed (status %d)\n", (int)p, status);
            failed = 1;
            for (pid_t q : pids)
                if (q != p) kill(q, SIGKILL);
        }
    }
    if (failed || !res->ok) return 4;
    FILE *f = std::fopen(a.out.c_str(), "w");
    if (!f) return 5;
    const int done = res->steps_done;
    double total = 0;
    for (int n = 0; n < done; n++) total += res->secs[n];
    std::fprintf(f, "{\"ranks\": %d, \"cells\": %lld, \"warmup\": %d, \"steps\": %d, \"steps_timed\": %d, "
                    "\"seconds\": %.9g, \"init_seconds\": %.6g, \"warmup_seconds\": %.6g, \"step_seconds\": [",
                 a.ranks, (long long)res->cells, a.warmup, a.steps, done, total, res->init_s, res->warmup_s);
    for (int n = 0; n < done; n++) std::fprintf(f, "%s%.9g", n ? ", " : "", res->secs[n]);
    std::fprintf(f, "], \"iterations\": [");
    for (int n = 0; n < done; n++) std::fprintf(f, "%s%lld", n ? ", " : "", (long long)res->it[n]);
    std::fprintf(f, "], \"residuals\": [");
    for (int n = 0; n < done; n++) std::fprintf(f, "%s%.17g", n ? ", " : "", res->err[n]);
    std::fprintf(f, "]}\n");
    std::fclose(f);
    return 0;
}
