/*
 * main.cxx -- triblock.exe, the drop-in for the reference's driver
 * (src/main.cxx:13-269):
 *
 *   triblock.exe <compute_mode> <device_id> <block_size> [options]
 *
 * Positional arguments as in the reference (src/main.cxx:38-55); only
 * compute_mode 2 (CUDA) runs.  Reads ./gpuline.mesh.data.bin and
 * ./gpuline.jacobian.data.bin, factors, runs the LIJ sweeps and prints the
 * reference's timing lines plus the per-sweep residual the reference lacks.
 *
 * Options (after the positional arguments):
 *   --iters N          fixed number of sweeps (default 30, src/main.cxx:20)
 *   --tol T            sweep until ||R||/||R0|| <= T instead (device-side test)
 *   --max-sweeps N     sweep limit with --tol (default 1000)
 *   --algo ref|fp64|mixed|pij   TBS_ALGO_* (default fp64; pij: point-implicit Jacobi)
 *   --inner M          FP32 inner sweeps per outer step for --algo mixed
 *   --gen L K SHIFT SEED    synthetic structured mesh + seeded Jacobian, at
 *                      the block size of the third positional argument
 *   --nrhs N           solve N right-hand sides together (tbs_solve_multi,
 *                      --algo fp64, to --tol): the Jacobian's rhs and N-1
 *                      seeded U(-1,1) vectors
 *   --gmres M          line-preconditioned GMRES(M) to --tol (tbs_gmres,
 *                      --algo fp64, one sweep per preconditioner step)
 *   --write-files      with --gen: also write the two data files to cwd
 *   --mesh PATH / --jac PATH   other input files
 *   --json             one JSON summary line at the end
 */
#include "Jacobian.hxx"
#include "Mesh.hxx"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cctype>
#include <cstring>
#include <string>

#define GREEN "\x1B[1;92m"
#define RED "\x1B[1;31m"
#define COLOR_OFF "\x1B[0m"

static double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

static void usage() {
    std::printf(
        "Arguments:\n"
        "  compute_mode: 0=Serial, 1=HIP, 2=CUDA, 3=OpenCL, 4=OpenMP, 5=DPC++, 6=Metal (apple)\n"
        "                (this build: 2=CUDA on sm_100a only)\n"
        "  device_id:    Device ID on node\n"
        "  block_size:   Size of the matrix sub-block (i.e., # of variables/eqns; e.g., 9x9 default)\n"
        "Options: --iters N | --tol T [--max-sweeps N] | --algo ref|fp64|mixed|pij | --inner M\n"
        "         --gen L K SHIFT SEED [--write-files] | --mesh PATH | --jac PATH | --json\n"
        "         --nrhs N (with --tol) | --gmres M (with --tol)\n");
}

int main(int argc, char **argv) {
    int compute_mode = TBS_CUDA_MODE, device_id = 0, block_size = 9, iters = 30;
    double tol = -1.0;
    int max_sweeps = 1000, algo = TBS_ALGO_FP64, inner = 4, nrhs = 1, gmres_m = 0;
    bool gen = false, write_files = false, json = false;
    int gL = 0, gK = 0;
    double gshift = 9.0;
    unsigned long long gseed = 0;
    std::string mesh_path = "gpuline.mesh.data.bin", jac_path = "gpuline.jacobian.data.bin";

    std::printf("+================================================================================+\n");
    std::printf(" >>>>         " GREEN "./triblock.exe" COLOR_OFF " <compute_mode> <device_id> <block_size>         <<<< \n");
    if (argc > 1 && (!std::strcmp(argv[1], "--help") || !std::strcmp(argv[1], "-help"))) {
        usage();
        std::printf("+================================================================================+\n");
        return 0;
    }
    int pos = 0;
    for (int a = 1; a < argc; ++a) {
        std::string s = argv[a];
        auto need = [&](int n) {
            if (a + n >= argc) {
                std::fprintf(stderr, RED "ERROR: %s needs %d value(s)" COLOR_OFF "\n", s.c_str(), n);
                std::exit(2);
            }
        };
        try {
            if (s == "--iters") { need(1); iters = std::stoi(argv[++a]); }
            else if (s == "--tol") { need(1); tol = std::stod(argv[++a]); }
            else if (s == "--max-sweeps") { need(1); max_sweeps = std::stoi(argv[++a]); }
            else if (s == "--inner") { need(1); inner = std::stoi(argv[++a]); }
            else if (s == "--nrhs") { need(1); nrhs = std::stoi(argv[++a]); }
            else if (s == "--gmres") { need(1); gmres_m = std::stoi(argv[++a]); }
            else if (s == "--algo") {
                need(1);
                std::string v = argv[++a];
                if (v == "ref") algo = TBS_ALGO_REFERENCE;
                else if (v == "fp64") algo = TBS_ALGO_FP64;
                else if (v == "mixed") algo = TBS_ALGO_MIXED;
                else if (v == "pij") algo = TBS_ALGO_PIJ;
                else { std::fprintf(stderr, RED "ERROR: unknown --algo %s" COLOR_OFF "\n", v.c_str()); return 2; }
            } else if (s == "--gen") {
                need(4);
                gen = true;
                gL = std::stoi(argv[++a]);
                gK = std::stoi(argv[++a]);
                gshift = std::stod(argv[++a]);
                gseed = std::stoull(argv[++a]);
            } else if (s == "--write-files") write_files = true;
            else if (s == "--mesh") { need(1); mesh_path = argv[++a]; }
            else if (s == "--jac") { need(1); jac_path = argv[++a]; }
            else if (s == "--json") json = true;
            else if (!s.empty() && s[0] == '-' && !(s.size() > 1 && std::isdigit((unsigned char)s[1]))) {
                std::fprintf(stderr, RED "ERROR: unknown option %s" COLOR_OFF "\n", s.c_str());
                usage();
                return 2;
            } else {
                const int v = std::stoi(s);
                if (pos == 0) compute_mode = v;
                else if (pos == 1) device_id = v;
                else if (pos == 2) block_size = v;
                ++pos;
            }
        } catch (const std::exception &) {
            std::fprintf(stderr, RED "ERROR: bad value for %s" COLOR_OFF "\n", s.c_str());
            return 2;
        }
    }
    const char *mode_name = compute_mode == 0 ? "SERIAL MODE" : compute_mode == 1 ? "HIP MODE"
                          : compute_mode == 2 ? "CUDA MODE" : compute_mode == 3 ? "OpenCL MODE"
                          : compute_mode == 4 ? "OpenMP MODE" : compute_mode == 5 ? "DPC++ MODE"
                          : compute_mode == 6 ? "Metal MODE" : "UNKNOWN";
    std::printf(" -------------------------------------------------------------------------------- \n");
    std::printf(GREEN " TRIDIAGONAL BLOCK SOLVER: " COLOR_OFF "Block size: " GREEN "%d" COLOR_OFF
                ", Compute mode: " GREEN "%s" COLOR_OFF ", Device ID: " GREEN "%d" COLOR_OFF "\n",
                block_size, mode_name, device_id);
    std::printf(" -------------------------------------------------------------------------------- \n");
    std::printf("    %s\n", tbs_version());
    std::printf("+================================================================================+\n");

    try {
        Platform gpu(compute_mode, device_id);

        Mesh mesh;
        Jacobian Jac;
        if (gen) {
            if (!mesh.fromStructured(gL, gK, block_size)) throw std::runtime_error(mesh.error);
        } else {
            std::printf("---------------------------------\n");
            std::printf(GREEN "Reading %s" COLOR_OFF "\n", mesh_path.c_str());
            if (!mesh.fromFile(mesh_path.c_str())) throw std::runtime_error(mesh.error);
        }
        std::printf("  Mesh Statistics:\n    nvar: %d\n    nelem: %d\n    nintface: %d\n"
                    "    eftot: %d\n    nline: %d\n    nlineelem: %d\n",
                    mesh.nvar, mesh.nelem, mesh.nintface, mesh.eftot, mesh.nline, mesh.nlineelem);
        std::printf("  Max Line Element count: %d\n", mesh.max_line_nelem);
        if (gen) {
            if (!Jac.fromGenerator(mesh, gshift, gseed)) throw std::runtime_error(Jac.error);
            if (write_files) {
                if (!mesh.toFile("gpuline.mesh.data.bin") || !Jac.toFile("gpuline.jacobian.data.bin"))
                    throw std::runtime_error(tbs_last_error(nullptr));
                std::printf("Wrote gpuline.mesh.data.bin and gpuline.jacobian.data.bin\n");
            }
        } else {
            std::printf(GREEN "Reading %s" COLOR_OFF "\n", jac_path.c_str());
            if (!Jac.fromFile(mesh.nlineelem, jac_path.c_str())) throw std::runtime_error(Jac.error);
        }
        std::printf("Read Jac Stats:\n  nvar: %d\n  nelem: %d\n  nintface: %d\n", Jac.nvar, Jac.nelem,
                    Jac.nintface);
        if (Jac.nelem != mesh.nelem || Jac.nintface != mesh.nintface || Jac.nvar != mesh.nvar)
            throw std::runtime_error("mesh and Jacobian headers disagree (nvar/nelem/nintface)");
        if (block_size != Jac.nvar) {
            /* the reference packs A before resizing (src/main.cxx:90-91) so its A
             * goes stale; here the blocks are resized first */
            std::printf("Resizing NVAR: old=%d new=%d ...", Jac.nvar, block_size);
            Jac.resizeBlockSize(block_size);
            mesh.nvar = block_size;
            std::printf(" done!\n");
        }
        Jac.assembleTriBlocks(mesh);

        mesh.setupDevice(gpu);
        mesh.toDevice();
        Jac.setupDevice(gpu);
        Jac.toDevice();
        std::printf("=========================================\n");
        std::printf("GPU Memory Allocated (MB): %g\n", gpu.memoryAllocated() / 1024. / 1024.);
        std::printf("=========================================\n");

        tbs_ctx *ctx = gpu.ctx;
        if (algo == TBS_ALGO_MIXED) tbs_set_inner_sweeps(ctx, inner);
        tbs_profile_enable(ctx, 1);
        double t0 = now_s();
        if (tbs_factor(ctx, algo) != TBS_OK) throw std::runtime_error(tbs_last_error(ctx));
        const double LU_time = now_s() - t0;
        std::printf("   LU Time: %f\n", LU_time);
        tbs_profile_reset(ctx);

        if ((nrhs > 1 || gmres_m > 0) && tol < 0.0)
            throw std::runtime_error("--nrhs and --gmres need --tol");
        std::vector<double> hist;
        int sweeps = 0;
        t0 = now_s();
        if (nrhs > 1) {
            /* the Jacobian's rhs, then seeded U(-1,1) vectors (splitmix64) */
            const size_t n = (size_t)mesh.nvar * mesh.nelem;
            std::vector<double> rhs(n * nrhs), U(n * nrhs);
            std::copy(Jac.rhs.begin(), Jac.rhs.end(), rhs.begin());
            unsigned long long z0 = gseed + 0x5EEDull;
            for (size_t t = n; t < rhs.size(); ++t) {
                unsigned long long z = (z0 += 0x9E3779B97F4A7C15ull);
                z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
                z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
                z ^= z >> 31;
                rhs[t] = (double)(z >> 11) * 0x1.0p-53 * 2.0 - 1.0;
            }
            std::vector<int> sw(nrhs);
            hist.assign((size_t)nrhs * (max_sweeps + 1), 0.0);
            if (tbs_solve_multi(ctx, nrhs, rhs.data(), U.data(), tol, max_sweeps, sw.data(), hist.data(),
                                max_sweeps + 1) != TBS_OK)
                throw std::runtime_error(tbs_last_error(ctx));
            for (int r = 0; r < nrhs; ++r) {
                const double *h = hist.data() + (size_t)r * (max_sweeps + 1);
                std::printf("  rhs %3d: %4d sweeps, ||R||/||R0|| = %.3e\n", r, sw[r],
                            h[0] > 0 ? h[sw[r]] / h[0] : 0.0);
            }
            hist.resize(max_sweeps + 1); /* right-hand side 0 in the report below */
            sweeps = sw[0];
        } else if (gmres_m > 0) {
            hist.assign((size_t)max_sweeps + 1, 0.0);
            if (tbs_gmres(ctx, gmres_m, 1, tol, max_sweeps, &sweeps, hist.data()) != TBS_OK)
                throw std::runtime_error(tbs_last_error(ctx));
            std::printf("  GMRES(%d): %d Arnoldi steps\n", gmres_m, sweeps);
        } else if (tol >= 0.0) {
            hist.assign((size_t)max_sweeps + 1, 0.0);
            if (tbs_solve(ctx, tol, max_sweeps, &sweeps, hist.data()) != TBS_OK)
                throw std::runtime_error(tbs_last_error(ctx));
            double tn = -1.0;
            int checks = 0, restarts = 0;
            if (tbs_solve_check(ctx, &tn, &checks, &restarts) == TBS_OK && checks > 0)
                std::printf("  true-residual check at convergence: %d check(s), %d restart(s), "
                            "||rhs + J U|| = %.10e\n", checks, restarts, tn);
        } else {
            hist.assign((size_t)iters + 1, 0.0);
            if (tbs_sweep(ctx, iters, hist.data()) != TBS_OK) throw std::runtime_error(tbs_last_error(ctx));
            sweeps = iters;
        }
        const double sweep_time = now_s() - t0;

        std::printf("-----------------------------------------\n");
        std::printf("  sweep     ||R||_2              ||R||/||R0||\n");
        for (int s = 0; s <= sweeps; ++s)
            std::printf("  %5d  %.10e  %.10e\n", s, hist[s], hist[0] > 0 ? hist[s] / hist[0] : 0.0);

        /* per-kernel device times */
        int nk = TBS_PROFILE_MAX;
        const char *names[TBS_PROFILE_MAX];
        long long launches[TBS_PROFILE_MAX];
        double ms[TBS_PROFILE_MAX];
        tbs_profile_read(ctx, &nk, names, launches, ms);
        std::printf("-----------------------------------------\n");
        double dev_ms = 0.0;
        for (int k = 0; k < nk; ++k) {
            double b = 0.0;
            const bool hasb = tbs_kernel_bytes(ctx, names[k], &b) == TBS_OK;
            dev_ms += ms[k];
            if (hasb && ms[k] > 0)
                std::printf("  %-14s %6lld launches %10.4f ms  %8.1f GB/s\n", names[k], launches[k], ms[k],
                            b * launches[k] / (ms[k] * 1e-3) / 1e9);
            else
                std::printf("  %-14s %6lld launches %10.4f ms\n", names[k], launches[k], ms[k]);
        }
        /* the reference's byte model, src/main.cxx:149-175, per sweep */
        const double N = mesh.nelem, F = mesh.nintface, nv = mesh.nvar;
        const double ints = 4.0 * (mesh.linesize.size() + mesh.linepoint.size() + mesh.lines.size() +
                                   mesh.lineface.size());
        const double du = 8.0 * (3 * nv * nv * N + 5 * nv * N) + ints;
        const double cp = 8.0 * 5 * nv * N;
        const double lr = 8.0 * (nv * nv * N + 2 * nv * nv * F + 5 * nv * N + 2 * nv * N) + ints +
                          4.0 * (mesh.epoint.size() + mesh.ef.size() + mesh.fc.size());
        const double refmodel = (du + cp + lr) * sweeps;
        std::printf("-----------------------------------------\n");
        std::printf("[b200] Sweeps: %d\n", sweeps);
        std::printf("[b200] Sweep Time: %f  (%.1f sweeps/s)\n", sweep_time, sweeps / sweep_time);
        std::printf("[b200] Device kernel time: %f  %.1f GB/s (reference byte model)\n", dev_ms * 1e-3,
                    dev_ms > 0 ? refmodel / (dev_ms * 1e-3) / 1e9 : 0.0);
        std::printf("[b200] Total Time: %f\n", sweep_time + LU_time);
        double tr = 0.0;
        tbs_true_residual_norm(ctx, &tr);
        std::printf("[b200] True residual ||rhs + J U||: %.10e  (relative %.3e)\n", tr,
                    hist[0] > 0 ? tr / hist[0] : 0.0);
        std::printf("-----------------------------------------\n");
        if (json) {
            std::printf("{\"nelem\": %d, \"nline\": %d, \"algo\": %d, \"sweeps\": %d, \"lu_s\": %.6f, "
                        "\"sweep_s\": %.6f, \"sweeps_per_s\": %.3f, \"rel_resid\": %.6e, "
                        "\"true_rel_resid\": %.6e}\n",
                        mesh.nelem, mesh.nline, algo, sweeps, LU_time, sweep_time, sweeps / sweep_time,
                        hist[0] > 0 ? hist[sweeps] / hist[0] : 0.0, hist[0] > 0 ? tr / hist[0] : 0.0);
        }
    } catch (const std::exception &ex) {
        std::fprintf(stderr, RED "ERROR: %s" COLOR_OFF "\n", ex.what());
        return 1;
    }
    return 0;
}
