// mph_main.cpp — command-line drop-in for the reference solver executable.
//
//   mph_b200 [data grid prof vtk log nthreads] [--dim=2|3] [--mode=fp64|mixed|mixed_p64]
//
// Same positional arguments and defaults as the reference's main()
// (main.cpp:293-307; nthreads is accepted and ignored: the step runs on the
// GPU).  The loop reproduces main.cpp:357-452: start-up VTK "output.vtk",
// then per step the .prof output test, the explicit step, the .vtk output test
// (with the virial stress) and Time += Dt.  The reference chooses 2-D/3-D at
// compile time (-D TWO_DIMENSIONAL); here --dim selects it, and an executable
// name ending in "_2d" defaults to 2-D.  Timing is wall clock (the reference's
// clock() sums CPU time over threads).
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>
#include "mph_b200.h"

static FILE* g_log = nullptr;

static void log_printf(const char* fmt, ...) {
    va_list a, b;
    va_start(a, fmt);
    va_copy(b, a);
    if (g_log) std::vfprintf(g_log, fmt, a);
    std::vfprintf(stderr, fmt, b);
    va_end(a);
    va_end(b);
}

static const char* status_text(int st) {
    switch (st) {
        case MPH_ERR_ARG: return "invalid argument";
        case MPH_ERR_IO: return "file could not be opened or parsed";
        case MPH_ERR_CUDA: return "CUDA runtime error";
        case MPH_ERR_CAPACITY: return "a device capacity was exceeded";
        case MPH_ERR_DEVICE: return "a device error flag was raised";
        case MPH_ERR_NONFINITE: return "NaN or Inf in the particle state";
        case MPH_ERR_STATE: return "call not valid in this state";
        case MPH_ERR_NOMEM: return "allocation failed";
        case MPH_ERR_GEOMETRY: return "cell grid incompatible with the radius";
        default: return "error";
    }
}

// Logs the failure (the library's message, else the status meaning) and ends.
static int die(mph_ctx* ctx, int st, const char* what, const char* path = nullptr) {
    char msg[512] = {0};
    mph_last_error(ctx, msg, sizeof(msg));
    log_printf("error %d in %s%s%s: %s\n", st, what, path ? " " : "", path ? path : "",
               msg[0] ? msg : status_text(st));
    if (ctx) mph_destroy(ctx);
    if (g_log) std::fclose(g_log);
    return 1;
}

int main(int argc, char** argv) {
    std::string data = "sample.data", grid = "sample.grid", prof = "sample%03d.prof", vtk = "sample%03d.vtk",
                logf = "sample.log";
    int dim = 3, mode = MPH_MODE_FP64;
    {
        const std::string exe = argv[0];
        if (exe.size() >= 3 && exe.compare(exe.size() - 3, 3, "_2d") == 0) dim = 2;
    }
    std::vector<std::string> pos;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if (a.rfind("--dim=", 0) == 0) dim = std::atoi(a.c_str() + 6);
        else if (a == "--mode=mixed") mode = MPH_MODE_MIXED;
        else if (a == "--mode=mixed_p64") mode = MPH_MODE_MIXED_P64;
        else if (a == "--mode=fp64") mode = MPH_MODE_FP64;
        else if (a.rfind("--", 0) == 0) {
            std::fprintf(stderr, "unknown option %s\nusage: %s [data grid prof vtk log nthreads] [--dim=2|3] "
                                 "[--mode=fp64|mixed|mixed_p64]\n", a.c_str(), argv[0]);
            return 2;
        } else pos.push_back(a);
    }
    if (pos.size() > 0) data = pos[0];
    if (pos.size() > 1) grid = pos[1];
    if (pos.size() > 2) prof = pos[2];
    if (pos.size() > 3) vtk = pos[3];
    if (pos.size() > 4) logf = pos[4];
    g_log = std::fopen(logf.c_str(), "w");
    if (!g_log) std::fprintf(stderr, "error in open %s\n", logf.c_str());
    {
        time_t t = time(NULL);
        log_printf("start reading files at %s\n", ctime(&t));
    }
    mph_params p;
    mph_params_defaults(&p);
    int bad = 0;
    int st = mph_read_data_file(data.c_str(), &p, &bad);
    if (st != MPH_OK) return die(nullptr, st, "reading the data file", data.c_str());
    if (bad) log_printf("%d invalid line(s) in data file \"%s\"\n", bad, data.c_str());
    mph_grid_header h;
    st = mph_read_grid_header(grid.c_str(), &h);
    if (st != MPH_OK) return die(nullptr, st, "reading the grid header", grid.c_str());
    std::vector<int> type(h.particle_count);
    std::vector<double> x(3 * (size_t)h.particle_count), v(3 * (size_t)h.particle_count);
    st = mph_read_grid_file(grid.c_str(), &h, h.particle_count, type.data(), x.data(), v.data());
    if (st != MPH_OK) return die(nullptr, st, "reading the grid file", grid.c_str());
    {
        time_t t = time(NULL);
        log_printf("start initialization at %s\n", ctime(&t));
    }
    mph_ctx* ctx = nullptr;
    st = mph_create(&p, &h, dim, mode, type.data(), x.data(), v.data(), &ctx);
    if (st != MPH_OK) return die(nullptr, st, "mph_create");
    mph_constants c;
    mph_get_constants(ctx, &c);
    log_printf("N0a = %e, count=%d\n", c.n0a, c.n0a_count);
    log_printf("N0p = %e, count=%d\n", c.n0p, c.n0p_count);
    log_printf("CellCount[DIM]: %d %d %d\n", c.cell_count[0], c.cell_count[1], c.cell_count[2]);
    log_printf("TotalCellCount: %d\n", c.total_cell_count);
    log_printf("CellWidth[DIM]: %e %e %e\n", c.cell_width[0], c.cell_width[1], c.cell_width[2]);
    mph_info info;
    mph_get_info(ctx, &info);
    log_printf("NeighborIndCount = %lld\n", info.neighbor_ind_count);
    st = mph_write_vtk(ctx, "output.vtk");
    if (st != MPH_OK) return die(ctx, st, "writing output.vtk");
    {
        time_t t = time(NULL);
        log_printf("start main roop at %s\n", ctime(&t));
    }
    double Time = h.time, OutputNext = 0.0, VtkOutputNext = 0.0;
    const double Dt = p.dt;
    int iStep = (int)(Time / Dt);
    long long steps = 0;
    double t_step = 0.0, t_out = 0.0;
    using clk = std::chrono::steady_clock;
    const auto t_begin = clk::now();
    char fname[1024];
    while (Time < p.end_time + 1.0e-5 * Dt) {
        if (Time + 1.0e-5 * Dt >= OutputNext) {
            const auto a = clk::now();
            std::snprintf(fname, sizeof(fname), prof.c_str(), iStep);
            st = mph_write_prof_async(ctx, fname);  // formatted now, written behind the next steps
            if (st != MPH_OK) return die(ctx, st, "writing a prof file");
            log_printf("@ Prof Output Time : %e\n", Time);
            OutputNext += p.output_interval;
            t_out += std::chrono::duration<double>(clk::now() - a).count();
        }
        // The step just checked always runs; the steps after it join the same
        // mph_step call while no output falls between them (no VTK after, no
        // prof before, the loop not ending), found by running the loop's own
        // Time additions and tests ahead.  One call of several steps keeps
        // the rebuild test on the device (step graphs).
        int k = 1;
        {
            double t = Time;
            while (k < 1000) {
                if (t + 1.0e-5 * Dt >= VtkOutputNext) break;  // a VTK after this step
                const double tn = t + Dt;
                if (!(tn < p.end_time + 1.0e-5 * Dt)) break;  // the loop ends after it
                if (tn + 1.0e-5 * Dt >= OutputNext) break;    // a prof before the next
                t = tn;
                ++k;
            }
        }
        const auto a = clk::now();
        st = mph_step(ctx, k);
        if (st == MPH_OK) st = mph_synchronize(ctx);
        if (st != MPH_OK) return die(ctx, st, "mph_step");
        t_step += std::chrono::duration<double>(clk::now() - a).count();
        steps += k;
        for (int s = 1; s < k; ++s) {  // the steps before the last: no output after them
            Time += Dt;
            ++iStep;
        }
        if (Time + 1.0e-5 * Dt >= VtkOutputNext) {
            const auto b = clk::now();
            st = mph_compute_virial(ctx);  // every form: VirialPressureAtParticle is a VTK field
            if (st != MPH_OK) return die(ctx, st, "virial");
            std::snprintf(fname, sizeof(fname), vtk.c_str(), iStep);
            st = mph_write_vtk_async(ctx, fname);
            if (st != MPH_OK) return die(ctx, st, "writing a vtk file");
            log_printf("@ Vtk Output Time : %e\n", Time);
            VtkOutputNext += p.vtk_output_interval;
            t_out += std::chrono::duration<double>(clk::now() - b).count();
        }
        Time += Dt;
        ++iStep;
    }
    {
        const auto a = clk::now();
        st = mph_output_wait(ctx);  // the files still being written behind the step
        if (st != MPH_OK) return die(ctx, st, "writing output files");
        t_out += std::chrono::duration<double>(clk::now() - a).count();
    }
    const double total = std::chrono::duration<double>(clk::now() - t_begin).count();
    mph_get_info(ctx, &info);
    {
        time_t t = time(NULL);
        log_printf("end main roop at %s\n", ctime(&t));
    }
    const int nf = info.fluid_particle_end - info.fluid_particle_begin;
    log_printf("steps:                   %lld (rebuilds %lld)\n", steps, info.rebuild_count);
    log_printf("explicit step:           %lf [wall sec]\n", t_step);
    log_printf("output:                  %lf [wall sec] (formatting on the device; file writes overlap the steps)\n",
               t_out);
    log_printf("total:                   %lf [wall sec]\n", total);
    if (t_step > 0)
        log_printf("particle-updates/s:      %e (fluid %d), %e (all %d)\n", nf * (double)steps / t_step, nf,
                   info.particle_count * (double)steps / t_step, info.particle_count);
    mph_destroy(ctx);
    if (g_log) std::fclose(g_log);
    return 0;
}
