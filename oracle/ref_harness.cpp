/*
 * ref_harness.cpp — drives the reference solver's own code in-process.
 *
 * TEST INFRASTRUCTURE ONLY (the checker and the CPU baseline, never the
 * product).  oracle/Makefile compiles this file with -I pointing at the
 * reference's source directory, so that source/main.cpp of
 * Masahiro-Kondo-AIST/MphExplicit is compiled unmodified from where it lies;
 * nothing of it is copied here.  Its `main` is renamed so this file can
 * provide the command line below, which calls the reference's own static
 * routines in the order of its main() (main.cpp:324-364 start-up,
 * main.cpp:386-431 + 449 per step) and dumps the reference's arrays.
 *
 *   ref_mph dump <data> <grid> <nsteps> <out.bin> [virial] [vtk=<path>] [prof=<path>]
 *   ref_mph time <data> <grid> <warmup> <steps> <threads> [max_seconds] [rebuild_at=<k>]
 *
 * The dump is a little-endian binary file:
 *   int32 magic 0x4d504852, int32 version 1, int32 n, int32 total_cell_count,
 *   int64 neighbor_ind_count, int64 rebuilds, double time,
 *   double n0a, double n0p, int32 cell_count[3], int32 fluid_begin,
 *   int32 fluid_end, int32 wall_begin, int32 wall_end, int32 pad,
 *   then arrays: pidx[n] i32, type[n] i32, x[n*3] f64, v[n*3] f64,
 *   force[n*3] f64, ncount[n] i32, densA[n] f64, strainP[n] f64, divP[n] f64,
 *   presP[n] f64, presA[n] f64, gc[n*3] f64, virialP[n] f64, cellIndex[n] i32,
 *   cfb[tot] cfe[tot] cwb[tot] cwe[tot] i32, nptr[n+1] i64, nind[nic] i32.
 */
#include <chrono>
#include <cstdint>
#include <string>
#include <vector>

#define main mph_reference_main
#include "main.cpp"
#undef main

static long long g_rebuilds = 0;
static bool g_force_rebuild = false;  // set by `time ... rebuild_at=<k>` for one step

static void startup(const char* data, const char* grid) {
    log_open("/dev/null");
    readDataFile((char*)data);
    readGridFile((char*)grid);
    initializeWeight();
    initializeFluid();
    initializeWall();
    initializeDomain();
    calculateCellParticle();
    calculateNeighbor();
    calculateDensityA();
    calculateGravityCenter();
    calculateDensityP();
}

static void one_step() {
    calculateConvection();
    calculateWall();
    calculatePeriodicBoundary();
    resetForce();
    // neighborCalculation() is always evaluated (its cost is part of every
    // step); a forced rebuild then runs the same three routines the loop runs
    // when the test fires (main.cpp:399-403).
    if (neighborCalculation() == 1 || g_force_rebuild) {
        g_force_rebuild = false;
        freeNeighbor();
        calculateCellParticle();
        calculateNeighbor();
        ++g_rebuilds;
    }
    calculateDensityA();
    calculateGravityCenter();
    calculateDensityP();
    calculateDivergenceP();
    calculatePhysicalCoefficients();
    calculatePressureP();
    calculatePressureA();
    calculateDiffuseInterface();
    calculateViscosityV();
    calculateGravity();
    calculateAcceleration();
    Time += Dt;
}

template <class T>
static void put(FILE* f, const T* p, size_t n) { fwrite(p, sizeof(T), n, f); }

static int cmd_dump(int argc, char** argv) {
    if (argc < 6) return 2;
    startup(argv[2], argv[3]);
    const int nsteps = atoi(argv[4]);
    for (int s = 0; s < nsteps; ++s) one_step();
    for (int a = 6; a < argc; ++a) {
        const std::string opt = argv[a];
        if (opt == "virial") calculateVirialStressAtParticle();
        else if (opt.rfind("vtk=", 0) == 0) writeVtkFile((char*)opt.c_str() + 4);     // main.cpp:698
        else if (opt.rfind("prof=", 0) == 0) writeProfFile((char*)opt.c_str() + 5);   // main.cpp:672
    }
    FILE* f = ::fopen(argv[5], "wb");
    if (!f) return 3;
    const int32_t hdr[4] = {0x4d504852, 1, ParticleCount, TotalCellCount};
    put(f, hdr, 4);
    const int64_t h64[2] = {(int64_t)NeighborIndCount, (int64_t)g_rebuilds};
    put(f, h64, 2);
    const double hd[3] = {Time, N0a, N0p};
    put(f, hd, 3);
    const int32_t hi[8] = {CellCount[0], CellCount[1], CellCount[2], FluidParticleBegin,
                           FluidParticleEnd, WallParticleBegin, WallParticleEnd, 0};
    put(f, hi, 8);
    const size_t n = ParticleCount;
    put(f, ParticleIndex, n);
    put(f, Property, n);
    put(f, &Position[0][0], 3 * n);
    put(f, &Velocity[0][0], 3 * n);
    put(f, &Force[0][0], 3 * n);
    put(f, NeighborCount, n);
    put(f, DensityA, n);
    put(f, VolStrainP, n);
    put(f, DivergenceP, n);
    put(f, PressureP, n);
    put(f, PressureA, n);
    put(f, &GravityCenter[0][0], 3 * n);
    put(f, VirialPressureAtParticle, n);
    put(f, CellIndex, n);
    put(f, CellFluidParticleBegin, (size_t)TotalCellCount);
    put(f, CellFluidParticleEnd, (size_t)TotalCellCount);
    put(f, CellWallParticleBegin, (size_t)TotalCellCount);
    put(f, CellWallParticleEnd, (size_t)TotalCellCount);
    std::vector<int64_t> ptr(n + 1);
    for (size_t i = 0; i <= n; ++i) ptr[i] = NeighborPtr[i];
    put(f, ptr.data(), n + 1);
    put(f, NeighborInd, (size_t)NeighborIndCount);
    ::fclose(f);
    return 0;
}

// time <data> <grid> <warmup> <steps> <threads> [max_seconds] [rebuild_at=<k>]
// Wall clock around the step loop only (start-up and warm-up excluded).
// max_seconds: stop after the step that crosses it.  rebuild_at=k: the k-th
// timed step (0-based) rebuilds the cell and neighbour lists whatever the
// displacement test says, so a short window holds the rebuild that the
// developed flow does every few tens of steps.
static int cmd_time(int argc, char** argv) {
    if (argc < 7) return 2;
    const int threads = atoi(argv[6]);
#ifdef _OPENMP
    omp_set_num_threads(threads > 0 ? threads : 1);
#endif
    double budget = 1.0e30;
    int rebuild_at = -1;
    for (int a = 7; a < argc; ++a) {
        const std::string opt = argv[a];
        if (opt.rfind("rebuild_at=", 0) == 0) rebuild_at = atoi(opt.c_str() + 11);
        else budget = atof(argv[a]);
    }
    const auto ts = std::chrono::steady_clock::now();
    startup(argv[2], argv[3]);
    const double startup_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - ts).count();
    const int warm = atoi(argv[4]), steps = atoi(argv[5]);
    for (int s = 0; s < warm; ++s) one_step();
    const long long rb0 = g_rebuilds;
    const auto t0 = std::chrono::steady_clock::now();
    int done = 0;
    double sec = 0.0;
    while (done < steps) {
        if (done == rebuild_at) g_force_rebuild = true;
        one_step();
        ++done;
        sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (sec > budget) break;
    }
    printf("{\"seconds\": %.9f, \"steps\": %d, \"particles\": %d, \"fluid\": %d, "
           "\"rebuilds\": %lld, \"threads\": %d, \"warmup\": %d, \"startup_seconds\": %.6f}\n",
           sec, done, ParticleCount, FluidParticleEnd - FluidParticleBegin, g_rebuilds - rb0, threads, warm,
           startup_s);
    return 0;
}

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    const std::string c = argv[1];
    if (c == "dump") return cmd_dump(argc, argv);
    if (c == "time") return cmd_time(argc, argv);
    return 2;
}
