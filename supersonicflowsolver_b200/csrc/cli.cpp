// psst_b200: command-line driver with the reference's inputs and outputs.
//
// Like main.cpp:9-63 it reads ./problem_manager (mesh file name, case name),
// the mesh and <case>.inp/.prop/.par|.sav/.bvp/.btq, then runs the iteration
// loop on the GPU and writes <case>_residual.dat (iteration, seconds, residual
// columns as psstFiniteVolumeGrid.cpp:369-396 prints them), <case>.sav
// (psstFiniteVolumeGrid.cpp:606-639) and the Fluent <case>.cas/<case>.dat
// (psstOutputManager.cpp) every iter_step iterations and at the end.
// Options: --precision 32|64, --jacobi (LocalAccTime1 from stage-start
// values), --no-renumber, --device N, --chunk N (iterations per launch batch).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "psst_b200.h"

static int die(const char *what) {
    std::fprintf(stderr, "%s: %s\n", what, psst_last_error());
    return 1;
}

static bool write_sav(const char *path, const psst_grid_info &gi, const std::vector<double> &prim,
                      const std::vector<int64_t> &zone, const std::vector<int64_t> &vbc, int64_t iter) {
    FILE *f = std::fopen(path, "w");
    if (!f) return false;
    const int dim = gi.dim;
    const int64_t nv = gi.nvol;
    std::fprintf(f, "%lld\n", (long long)iter);
    int64_t v = 0;
    while (v < nv) {  // bc 1 zones in ascending id (private_save_solution, :606-639)
        int64_t e = v;
        while (e < nv && zone[e] == zone[v]) ++e;
        if (vbc[v] == 1) {
            std::fprintf(f, "%lld\n%lld\n", (long long)zone[v], (long long)(e - v));
            for (int64_t i = v; i < e; ++i) {
                std::fprintf(f, "%.11f %.11f ", prim[i], prim[nv + i]);
                for (int k = 0; k < dim; ++k) std::fprintf(f, "%.11f ", prim[(2 + k) * nv + i]);
                std::fprintf(f, "\n");
            }
        }
        v = e;
    }
    std::fprintf(f, "0");
    std::fclose(f);
    return true;
}

int main(int argc, char **argv) {
    int precision = 64, jacobi = 0, renumber = 1, device = 0, chunk = 1000;
    for (int i = 1; i < argc; ++i) {
        if (!std::strcmp(argv[i], "--precision") && i + 1 < argc)
            precision = std::atoi(argv[++i]);
        else if (!std::strcmp(argv[i], "--jacobi"))
            jacobi = 1;
        else if (!std::strcmp(argv[i], "--no-renumber"))
            renumber = 0;
        else if (!std::strcmp(argv[i], "--device") && i + 1 < argc)
            device = std::atoi(argv[++i]);
        else if (!std::strcmp(argv[i], "--chunk") && i + 1 < argc)
            chunk = std::max(1, std::atoi(argv[++i]));
    }
    FILE *pm = std::fopen("problem_manager", "r");
    if (!pm) {
        std::fprintf(stderr, "Error: Could not open problem_manager file!");
        return 1;
    }
    char mesh[1024], cs[1024];
    if (std::fscanf(pm, "%1023s %1023s", mesh, cs) != 2) {
        std::fclose(pm);
        return 1;
    }
    std::fclose(pm);
    psst_grid *g = nullptr;
    if (psst_grid_read_fluent(mesh, &g)) return die("mesh");
    psst_grid_info gi;
    psst_grid_get_info(g, &gi);
    psst_scheme sc;
    std::vector<double> prim((size_t)(2 + gi.dim) * gi.nvol);
    if (psst_case_read(g, ".", cs, &sc, prim.data())) return die("case");
    sc.precision = precision;
    sc.lc1_mode = jacobi ? PSST_LC1_JACOBI : PSST_LC1_SEQUENTIAL;
    sc.renumber = renumber;
    psst_solver *s = nullptr;
    if (psst_solver_create(g, &sc, device, &s)) return die("solver");
    if (psst_solver_set_state(s, prim.data())) return die("state");
    std::vector<int64_t> zone(gi.nvol), vbc(gi.nvol);
    psst_grid_get_array(g, "vol_zone", zone.data(), gi.nvol);
    psst_grid_get_array(g, "vol_bc", vbc.data(), gi.nvol);
    const int nvv = gi.dim + 2;
    std::vector<double> rho(gi.nvol);
    const std::string resname = std::string(cs) + "_residual.dat", savname = std::string(cs) + ".sav";
    FILE *rf = std::fopen(resname.c_str(), sc.iter == 1 ? "w" : "a");
    if (!rf) return die("residual file");
    const auto t0 = std::chrono::steady_clock::now();
    int64_t it = sc.iter;
    while (it <= sc.max_iter) {
        int n = (int)std::min<int64_t>(chunk, sc.max_iter - it + 1);
        if (sc.iter_step > 0) n = (int)std::min<int64_t>(n, sc.iter_step - (it - 1) % sc.iter_step);
        std::vector<double> li((size_t)n * nvv);
        if (psst_explicit_solve(s, n, li.data(), nullptr)) return die("solve");
        const double sec =
            std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - t0).count() / 1000.0;
        for (int i = 0; i < n; ++i, ++it) {
            std::fprintf(rf, "%lld %.11e ", (long long)it, sec);
            for (int j = 0; j < nvv; ++j) std::fprintf(rf, " %.3e", li[(size_t)i * nvv + j]);
            std::fprintf(rf, "\n");
            if (sc.iter_step > 0 && it % sc.iter_step == 0) {
                psst_solver_get_state(s, prim.data(), nullptr);
                psst_solver_get_array(s, "rho", rho.data(), gi.nvol);
                if (psst_write_fluent(g, prim.data(), rho.data(), cs)) return die("output");
                write_sav(savname.c_str(), gi, prim, zone, vbc, it);
            }
        }
    }
    std::fclose(rf);
    psst_solver_get_state(s, prim.data(), nullptr);
    psst_solver_get_array(s, "rho", rho.data(), gi.nvol);
    if (psst_write_fluent(g, prim.data(), rho.data(), cs)) return die("output");
    write_sav(savname.c_str(), gi, prim, zone, vbc, psst_solver_iter(s));
    psst_solver_destroy(s);
    psst_grid_free(g);
    return 0;
}
