/*
 * mph_b200.h — C ABI of the B200 (sm_100a) MPH-WC explicit time step.
 *
 * The reference solver (Masahiro-Kondo-AIST/MphExplicit) is one C++ program whose
 * state lives in file-scope statics of source/main.cpp and whose step is the body
 * of the while loop at source/main.cpp:374-452.  It has no library interface; the
 * replaceable units are its file readers/writers, its set-up routines and the
 * per-step call sequence.  Each entry point below names the reference routine(s)
 * it replaces.  All entry points:
 *   - take plain host pointers and sizes (no device or framework types);
 *   - return an int status (MPH_OK == 0, negative on error) and never exit();
 *   - copy what they are given: the caller owns host buffers, the library owns
 *     device memory.
 * A context is used by one host thread at a time.  Work is ordered on one CUDA
 * stream per context; functions that return host data synchronise that stream.
 *
 * Particle arrays are "double[n][3]" (x,y,z per particle) as in the reference
 * (DIM is 3 even in 2-D, main.cpp:40).  Types 0/1 are fluid, 2/3 are wall
 * (main.cpp:43-47).
 */
#ifndef MPH_B200_H
#define MPH_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define MPH_TYPE_COUNT 4

/* ---- status codes ---------------------------------------------------- */
#define MPH_OK               0
#define MPH_ERR_ARG         -1   /* invalid argument                        */
#define MPH_ERR_IO          -2   /* file could not be opened / parsed       */
#define MPH_ERR_CUDA        -3   /* CUDA runtime error                      */
#define MPH_ERR_CAPACITY    -4   /* a device-side capacity was exceeded     */
#define MPH_ERR_DEVICE      -5   /* device-side error flag was raised       */
#define MPH_ERR_NONFINITE   -6   /* NaN/Inf detected in the particle state  */
#define MPH_ERR_STATE       -7   /* call not valid in the context's state   */
#define MPH_ERR_NOMEM       -8   /* host or device allocation failed        */
#define MPH_ERR_GEOMETRY    -9   /* cell grid incompatible with the radius  */

/* ---- step forms ------------------------------------------------------ */
/* Plain FP64 in the reference's operation order: bitonic cell sort, Verlet
 * neighbour list in the reference order, every pair sum in list order, no FMA
 * contraction.  Results are bit-identical to the reference's x86-64 build. */
#define MPH_MODE_FP64     0
/* FP32 pair arithmetic on cell-relative coordinates (exact FP32
 * displacements from hi/lo parts), compensated per-particle sums, FP64
 * position/velocity integration; its own counting-sort cell list and a
 * neighbour table with the short-range pairs first, rebuilt on the
 * reference's displacement criterion.  The DensityP terms, whose sum minus
 * N0p is the strain, are carried as double-float pairs of FP32 numbers (FP32
 * operations only): relative L2 velocity error vs FP64 ~3e-6 after 1000 steps
 * of the 2.78 M-particle dam break, against 6e-4 with plain FP32 terms. */
#define MPH_MODE_MIXED    1
/* The mixed form with the density sweep's pressure pairs (DensityP and
 * DivergenceP, which set the PressureP values) in FP64 and every force pair in
 * FP32: the FP32 strain sum carries ~1e-7 absolute error, which the bulk
 * modulus turns into pressure noise, while FP32 force pairs do not limit the
 * accuracy (relative L2 velocity error vs FP64 ~3e-6 after 1000 steps of the
 * 2.78 M-particle dam break, the same as MPH_MODE_MIXED's, whose density
 * sweep is faster). */
#define MPH_MODE_MIXED_P64 2
/* Flag for MPH_MODE_MIXED / MPH_MODE_MIXED_P64 (mode | MPH_MIXED_CELL_WALK):
 * the force sweep reads no neighbour table: one warp per cell walks the 3^D
 * stencil, keeps the candidates within the largest force radius of the box
 * around its own particles, stages them in shared memory and evaluates each
 * against every particle of the warp.  Same pair terms as the table sweep
 * (within the same accuracy bound); the density sweep still reads the short
 * part of the table. */
#define MPH_MIXED_CELL_WALK 0x100
/* The FP64 form with the viscosity and surface-tension pair terms
 * (ViscosityV main.cpp:1941-1985, DiffuseInterface :1778-1829, PressureA
 * force :1742-1775) replaced by an edge-MLP surrogate (mph_model) evaluated on
 * the tensor cores.  Every judge_interval steps the plain FP64 step is run
 * from the same state as the judge; when the relative L2 error of the
 * replaced terms (see mph_set_learned) exceeds the tolerance, that step and
 * the steps up to the next judgement take the plain step (fallback).  No
 * reference counterpart. */
#define MPH_MODE_LEARNED  3

/* ---- parameters read from the *.data file (main.cpp:489-539) --------- */
typedef struct mph_params {
    double dt;                                   /* Dt                       */
    double output_interval;                      /* OutputInterval           */
    double vtk_output_interval;                  /* VtkOutputInterval        */
    double end_time;                             /* EndTime                  */
    double radius_ratio_a;                       /* RadiusRatioA (= ratio G) */
    double radius_ratio_p;                       /* RadiusRatioP             */
    double radius_ratio_v;                       /* RadiusRatioV             */
    double density[MPH_TYPE_COUNT];
    double bulk_modulus[MPH_TYPE_COUNT];
    double bulk_viscosity[MPH_TYPE_COUNT];
    double shear_viscosity[MPH_TYPE_COUNT];
    double surface_tension[MPH_TYPE_COUNT];
    double interaction_ratio[MPH_TYPE_COUNT][MPH_TYPE_COUNT];
    double gravity[3];
    double wall_center[MPH_TYPE_COUNT][3];       /* rows 2 and 3 are used    */
    double wall_velocity[MPH_TYPE_COUNT][3];
    double wall_omega[MPH_TYPE_COUNT][3];
} mph_params;

/* ---- first two lines of a *.grid / *.prof file (main.cpp:549-557) ---- */
typedef struct mph_grid_header {
    double time;
    int    particle_count;
    double particle_spacing;
    double domain_min[3];
    double domain_max[3];
} mph_grid_header;

/* ---- derived constants (initializeWeight/Fluid/Domain, main.cpp:836-1084) */
typedef struct mph_constants {
    int    dim;
    double particle_volume;
    double radius_a, radius_g, radius_p, radius_v, max_radius;
    double swa, swg, swp, swv, n0a, n0p, r2g;
    int    n0a_count, n0p_count;
    double cof_k, cof_a[MPH_TYPE_COUNT];
    double domain_width[3];
    int    cell_count[3];
    int    total_cell_count;
    double cell_width[3];
    double wall_rotation[MPH_TYPE_COUNT][3][3];
} mph_constants;

/* ---- run-time counters of a context --------------------------------- */
typedef struct mph_info {
    int       particle_count;
    int       fluid_particle_begin, fluid_particle_end;   /* sorted order      */
    int       wall_particle_begin, wall_particle_end;
    long long neighbor_ind_count;     /* NeighborIndCount (FP64 form)          */
    int       max_neighbor_count;     /* longest neighbour list                */
    int       neighbor_capacity;      /* allocated list length per particle    */
    long long step;                   /* steps taken since mph_create          */
    long long rebuild_count;          /* neighbour rebuilds inside mph_step    */
    double    time;                   /* Time                                  */
    int       mode;
} mph_info;

typedef struct mph_ctx mph_ctx;

/* Zero/neutral parameters, matching the reference statics before
 * readDataFile runs (Dt = 1e100, everything else 0; main.cpp:56-211). */
int mph_params_defaults(mph_params* p);

/* Parse a *.data file.  Replaces readDataFile (main.cpp:489-539): same keys,
 * same sscanf patterns, '#' lines skipped, unknown lines counted in
 * *invalid_lines (may be NULL).  Returns MPH_ERR_IO if the file cannot be
 * opened (the reference would crash in fclose(NULL)). */
int mph_read_data_file(const char* path, mph_params* p, int* invalid_lines);

/* Read the two header lines of a *.grid / *.prof file (main.cpp:549-557). */
int mph_read_grid_header(const char* path, mph_grid_header* h);

/* Read a *.grid / *.prof file into caller arrays of `capacity` particles.
 * Replaces the parsing part of readGridFile (main.cpp:541-640).  A file with
 * fewer particle lines than its header announces returns MPH_ERR_IO (the
 * reference silently leaves the rest uninitialised). */
int mph_read_grid_file(const char* path, mph_grid_header* h, int capacity,
                       int* type, double* xyz, double* vel);

/* Write a *.grid / *.prof file.  Same format as writeProfFile
 * (main.cpp:672-696) and the generator (generator/generator.cpp:197-217 uses
 * "%lf" for time; this writer uses the solver's "%e"). */
int mph_write_grid_file(const char* path, const mph_grid_header* h,
                        const int* type, const double* xyz, const double* vel);

/* ---- the scene generator (generator/generator.cpp) --------------------
 * The reference's pre-processor GeneratorForMph reads a *.boid list of
 * cuboids and writes a *.grid with particles on each cuboid's lattice.  These
 * entry points replace it; on valid input the *.grid bytes are the
 * reference's.  Malformed input returns MPH_ERR_IO with the reason (read it
 * with mph_generator_last_error), where the reference prints a message and
 * goes on, or never returns (a cuboid without EndCuboid). */
typedef struct mph_cuboid {
    double spacing;        /* Spacing                                  */
    int type;              /* Type (0/1 fluid, 2/3 wall)               */
    double lower[3];       /* Lower                                    */
    double upper[3];       /* Upper                                    */
    double velocity[3];    /* Velocity                                 */
} mph_cuboid;

typedef struct mph_boid {
    double particle_distance;  /* ParticleDistance (the *.grid's l0)   */
    double lower_domain[3];    /* LowerDomain                          */
    double upper_domain[3];    /* UpperDomain                          */
    int cuboid_count;
} mph_boid;

/* Read a *.boid file (readfile + readCuboid, generator.cpp:49-164): up to
 * `capacity` cuboids are stored, *count receives how many the file holds
 * (MPH_ERR_CAPACITY when that is more than capacity; capacity 0 with
 * cuboids NULL asks for the count). */
int mph_read_boid_file(const char* path, mph_boid* boid, mph_cuboid* cuboids, int capacity, int* count);

/* Particles of the cuboids' lattices in the reference's order (genparticle,
 * generator.cpp:170-193: per cuboid, count = round(width/Spacing) per axis,
 * spacing = width/count, coordinates by repeated addition from lower +
 * spacing/2 while below upper - 0.49 spacing, x outermost).  With type, xyz or
 * vel NULL only *n is computed; otherwise up to `capacity` particles are
 * written (MPH_ERR_CAPACITY beyond). */
int mph_generate_cuboids(const mph_cuboid* cuboids, int count, int* type, double* xyz, double* vel,
                         long long capacity, long long* n);

/* Write generated particles as the generator's writefile does
 * (generator.cpp:197-217: time "%lf", then the header and particle lines). */
int mph_write_generated_grid(const char* path, const mph_boid* boid, long long n, const int* type,
                             const double* xyz, const double* vel);

/* The whole generator: read boid_path, write grid_path (GeneratorForMph
 * <stem> reads <stem>.boid and writes <stem>.grid, generator.cpp:37-47). */
int mph_generate_grid_file(const char* boid_path, const char* grid_path, long long* particle_count);

/* Message of the last failed generator call on this thread. */
int mph_generator_last_error(char* buf, int len);

/* Compute the derived constants without creating a context (initializeWeight,
 * initializeFluid's CofK/CofA, initializeWall, initializeDomain). dim is 2 or 3. */
int mph_compute_constants(const mph_params* p, const mph_grid_header* h, int dim,
                          mph_constants* c);

/* Create a context on the current CUDA device: copy the particles in, run the
 * set-up (main.cpp:330-333), the initial cell sort and neighbour list
 * (main.cpp:358-359) and the initial densities (main.cpp:362-364).
 * `type`, `xyz`, `vel` are in file order. */
int mph_create(const mph_params* p, const mph_grid_header* h, int dim, int mode,
               const int* type, const double* xyz, const double* vel,
               mph_ctx** out);

/* Advance nsteps explicit steps: the loop body main.cpp:386-431 plus
 * Time += Dt (main.cpp:449).  No file output.  Returns when the steps are
 * done.  Several FP64 steps run as one CUDA graph launch each, whose
 * conditional nodes make the neighbour-rebuild test (in the move kernel's
 * last block) and check a rebuilt list against its table on the device, with
 * no host round trip until the end: the same kernels, so the same bits.  A
 * list that outgrows its table ends the graph launches after that step's
 * reorder; the host grows the table and finishes the steps.  One step, the
 * mixed and learned forms, profiling on (mph_profile_enable), or graphs off:
 * the host reads the rebuild flag after each step's move. */
int mph_step(mph_ctx* ctx, int nsteps);

/* enable == 0: mph_step takes the host path for every step; 1 (the
 * default): graph launches for several FP64 steps.  Measured on one B200:
 * 0.036 against 0.040 ms per step on a 1,600-particle droplet, 2-3 % on
 * 10-20 k particles, within 1 % at 0.1-2.8 M particles. */
int mph_set_step_graphs(mph_ctx* ctx, int enable);

/* The FP64 (and learned) form's pair sweeps: 0 (the default) by size, one
 * warp per particle up to 40,000 particles in 3-D and 20,000 in 2-D, one
 * thread per particle above; 1 always a thread per particle; 2 always a warp
 * per particle.  The same bits either way (the warp's lanes compute the terms
 * of 32 list entries, one lane per sum adds them in list order). */
int mph_set_sweep_layout(mph_ctx* ctx, int layout);

/* Wait for the context's stream and report any device-side error flag. */
int mph_synchronize(mph_ctx* ctx);

int mph_get_info(mph_ctx* ctx, mph_info* info);
int mph_get_constants(mph_ctx* ctx, mph_constants* c);

/* Copy the current particle state to host arrays, in the context's current
 * (cell-sorted) order, as the reference's arrays are after a step.  Any pointer
 * may be NULL.  particle_index[i] is the file-order id of slot i
 * (ParticleIndex, main.cpp:75).  virial_pressure is valid after
 * mph_compute_virial.  Values the step itself does not need (DensityA without
 * surface tension, the walls' Force) are computed on the first read after a
 * step, from the arrays that step used: the same values as computing them in
 * the step, at the cost of a launch in this call. */
int mph_get_state(mph_ctx* ctx, int* particle_index, int* type,
                  double* xyz, double* vel, double* force, int* neighbor_count,
                  double* density_a, double* vol_strain_p, double* virial_pressure);

/* Overwrite positions and velocities (same sorted order as mph_get_state).
 * Used by callers that keep the state on the host between steps. */
int mph_set_state(mph_ctx* ctx, const double* xyz, const double* vel);

/* mph_step(ctx, nsteps), then the positions and velocities after the last
 * step into xyz[n][3] and vel[n][3] (sorted order; either may be NULL): the
 * same values as mph_step + mph_get_state, for callers that read the state
 * every step (main.cpp:404-431 writes it at output times).  In the FP64 form
 * the copies overlap the last step: the positions are final once its move
 * and any list rebuild are done and are copied while the sweeps run; when
 * vel is pinned and mapped (cudaHostAlloc memory, or cudaHostRegister with
 * cudaHostRegisterMapped) the force sweep stores each new velocity into it
 * directly as it computes it.  Pageable buffers give the same values with
 * less overlap.  The other forms step, then copy.  Returns after the copies
 * have landed. */
int mph_step_read_state(mph_ctx* ctx, int nsteps, double* xyz, double* vel);

/* Secondary per-particle fields in sorted order (any pointer may be NULL):
 * DivergenceP, PressureP, PressureA, GravityCenter[3]. */
int mph_get_fields(mph_ctx* ctx, double* divergence_p, double* pressure_p,
                   double* pressure_a, double* gravity_center);

/* Cell data of the last rebuild (FP64 form): CellIndex per sorted slot and
 * the per-cell fluid/wall particle ranges (main.cpp:1160-1247).  Arrays of
 * particle_count and total_cell_count entries; any pointer may be NULL. */
int mph_get_cells(mph_ctx* ctx, int* cell_index, int* fluid_begin, int* fluid_end,
                  int* wall_begin, int* wall_end);

/* The neighbour list of the last rebuild in CSR form (NeighborPtr /
 * NeighborInd, main.cpp:1452-1585): ptr has particle_count+1 entries, ind has
 * neighbor_ind_count entries.  FP64 form only. */
int mph_get_neighbors(mph_ctx* ctx, long long* ptr, int* ind, long long ind_capacity);

/* Virial stress and pressure at particles (calculateVirialStressAtParticle,
 * main.cpp:2057-2302), computed on the device from the current state: in the
 * reference's FP64 order for MPH_MODE_FP64 / MPH_MODE_LEARNED (bit-identical),
 * with FP32 pair terms over the form's own neighbour table for the mixed
 * forms (output only; close to the FP64 values, not equal). */
int mph_compute_virial(mph_ctx* ctx);

/* Output files in the reference formats and in sorted order:
 * writeVtkFile (main.cpp:698-834) and writeProfFile (main.cpp:672-696),
 * byte for byte.  The device formats every particle's lines ("%e" exact to
 * the last digit, as glibc prints it); the host copies the text out and writes
 * it.  These two return once the file is written. */
int mph_write_vtk(mph_ctx* ctx, const char* path);
int mph_write_prof(mph_ctx* ctx, const char* path);

/* The same files written behind the step: the state at the call is
 * formatted on the context's stream (ordered before any later mph_step), and a
 * writer thread of the context copies it out and writes the file while the
 * caller steps on.  Two documents can be in flight; a third call waits for the
 * first one's copy.  mph_output_wait returns once every file is written, with
 * the first write failure since the previous wait; mph_destroy also waits. */
int mph_write_vtk_async(mph_ctx* ctx, const char* path);
int mph_write_prof_async(mph_ctx* ctx, const char* path);
int mph_output_wait(mph_ctx* ctx);

/* The device formatter on its own: values[0..n) as "%e\n" lines, each value
 * first cast to float when as_float (writeVtkFile's "(float)" fields), into
 * out[0..capacity); *length = bytes written.  MPH_ERR_CAPACITY if out is too
 * small (at most 15 bytes per value). */
int mph_format_e(const double* values, long long n, int as_float, char* out, long long capacity,
                 long long* length);

/* writeVtkFile (main.cpp:698-834) from caller host arrays of n particles
 * (no context needed): same text, same field order, same float casts. */
int mph_write_vtk_arrays(const char* path, int n, const int* type, const double* xyz,
                         const double* vel, const double* force, const int* neighbor_count,
                         const double* density_a, const double* vol_strain_p,
                         const double* virial_pressure);

/* Mass, momentum and kinetic energy of the fluid, summed in FP64 on the
 * device (diagnostic of the mixed form).  out[0]=mass, out[1..3]=momentum,
 * out[4]=kinetic energy. */
int mph_conserved_sums(mph_ctx* ctx, double out[5]);

/* ---- exact checkpoint (no reference counterpart: the reference restarts from
 * a *.prof file, readGridFile main.cpp:541-640 with iStep = Time/Dt at :371,
 * whose "%e" text keeps ~7 digits and drops the moving walls' centres) -----
 * The file holds Time (in the grid header), the step count, the parameters
 * with Wall2/3 Center set to the centres reached, and every particle's type,
 * ParticleIndex, position and velocity in FP64, in the context's current
 * (cell-sorted) order -- the order of the *.prof file the reference would
 * write at that time.  Creating a context from it (mph_create with the
 * returned arrays) is the reference's restart from that *.prof, exactly. */
int mph_write_checkpoint(mph_ctx* ctx, const char* path);
/* The same file from host arrays (no GPU). */
int mph_write_checkpoint_arrays(const char* path, const mph_params* p, const mph_grid_header* h, int dim,
                                long long step, const int* type, const int* particle_index,
                                const double* xyz, const double* vel);
/* Parameters, grid header (Time, particle count, domain), dimension and step. */
int mph_read_checkpoint_header(const char* path, mph_params* p, mph_grid_header* h, int* dim, long long* step);
/* Everything, particles into caller arrays of `capacity` particles;
 * MPH_ERR_IO for a missing, foreign or truncated file. */
int mph_read_checkpoint(const char* path, mph_params* p, mph_grid_header* h, int* dim, long long* step,
                        int capacity, int* type, int* particle_index, double* xyz, double* vel);

/* ---- measurement hooks (no reference counterpart: the reference only has
 * clock() totals, main.cpp:287-288, 456-465) ---------------------------- */

/* The CUDA stream (cudaStream_t) all work of ctx is ordered on, so a caller
 * can record its own CUDA events around mph_step. */
void* mph_stream(mph_ctx* ctx);

/* Kernels launched by ctx since mph_create. */
long long mph_launch_count(mph_ctx* ctx);

typedef struct mph_kernel_stat {
    char      name[32];
    long long launches;
    double    total_ms;   /* sum of CUDA-event durations on the ctx stream */
} mph_kernel_stat;

/* enable != 0: from now on bracket every kernel launch with CUDA events on
 * the context's stream (statistics are reset).  enable == 0: stop. */
int mph_profile_enable(mph_ctx* ctx, int enable);

/* Synchronise and return the per-kernel statistics gathered since the last
 * mph_profile_enable(ctx, 1); *count receives the number of kernel names. */
int mph_profile_read(mph_ctx* ctx, mph_kernel_stat* out, int capacity, int* count);

/* Self-check of the exactly rounded FP64 division the FP64 kernels use in
 * place of the IEEE '/' (no reference counterpart): compares it bit for bit
 * with the hardware division on n random and adversarial operand pairs on the
 * current device; *mismatches receives the count (0 expected) and, if any,
 * first[0]/first[1] one failing numerator/denominator (may be NULL). */
int mph_check_exact_division(long long n, unsigned long long seed, long long* mismatches, double* first);

/* Cell sort without any allocation.  No counterpart in the reference: it is
 * for callers that cannot call cudaMalloc -- their device memory belongs to
 * another allocator (a framework's caching allocator, a pool with a fixed
 * budget) or they run a time-critical loop where allocating, and cudaFree's
 * device synchronisation, are not allowed.  It computes what the reference's
 * calculateCellParticle computes (main.cpp:1111-1247) for n particles in file
 * order: the sorted CellIndex (cell_index[n]), the bitonic permutation
 * CellParticle (cell_particle[n]) and the per-cell ranges as
 * cell_start[2*total_cell_count+1] (number of sorted keys below each key value:
 * fluid cell c spans [cell_start[c], cell_start[c+1]), wall cell c spans
 * [cell_start[c+T], cell_start[c+T+1]) with T = total_cell_count).
 * xyz (double[n][3]), type, and the three outputs are DEVICE pointers owned by
 * the caller; c comes from mph_compute_constants, h gives the domain origin;
 * stream is a cudaStream_t (NULL: the legacy default stream) and the call is
 * asynchronous on it.  The sort's scratch is a fixed static device array of
 * 2^21 ints (8 MiB), so n must be below 2^20 (1,048,576); larger n returns
 * MPH_ERR_CAPACITY.  Each call looks up that array's device address in the
 * current context (no allocation once the module is loaded); under CUDA's
 * lazy module loading (the default) the first call on a device, or the first
 * after a device reset, is the one that loads the library's module, and with
 * it the 8 MiB array, onto that device, which then holds it until the process
 * exits (or the next reset).  Callers with a fixed device budget should
 * therefore make the first call during their own set-up, and before any
 * stream capture.  All calls share the one
 * scratch array: calls that overlap on the GPU (other streams, other host
 * threads) race and must be serialised by the caller.  Allocates nothing
 * (no cudaMalloc, cudaFree or allocating library call). */
int mph_cell_sort_noalloc(const mph_constants* c, const mph_grid_header* h, int n,
                          const double* xyz, const int* type, int* cell_index,
                          int* cell_particle, int* cell_start, void* stream);

/* ---- learned form: edge-MLP surrogate (no reference counterpart) ------
 * Network: 9 inputs -> 128 -> 128 -> 128 -> 3, SiLU, BF16 weights and
 * activations, FP32 accumulation, trained and evaluated by the library's own
 * tcgen05 kernels.  Inputs of edge (i, j): (x_j - x_i)/l0 (3), (v_j - v_i) /
 * velocity_scale (3), |x_j - x_i|/l0, type_i, type_j.  Output: the pair's
 * viscous + surface-tension force on i / force_scale.
 * A sample is MPH_SAMPLE_FLOATS floats: (dx, dy, dz, r)/l0,
 * (ux, uy, uz, type_i + 4*type_j), (fx, fy, fz, valid) with f the FP64 pair
 * term in N.  Parameters are the flat FP32 vector W1[128][16], b1[128],
 * W2[128][128], b2, W3[128][128], b3, W4[16][128], b4[16] (W[out][in]; input
 * columns >= 9 and output rows >= 3 are padding and stay zero). */
#define MPH_SAMPLE_FLOATS 12
typedef struct mph_model mph_model;
typedef struct mph_dataset mph_dataset;

/* Self-test of the bounded tensor-core waits (no reference counterpart).
 * Every mbarrier wait of the edge-MLP kernels gives up after a fixed number
 * of polls (about a second), sets the model's error flag, waits (within the
 * same limit) for any MMA group still in flight and frees its tensor memory
 * before the kernel returns; the call then reports MPH_ERR_DEVICE.  This entry
 * point runs the training (kernel 0) or inference (kernel 1) kernel on one
 * tile with its MMA groups withheld and a limit of `polls` (1 .. 2^22), so
 * the first wait runs out with nothing in flight.  It returns that
 * MPH_ERR_DEVICE and clears the flag again: the model stays usable. */
int mph_model_check_wait(mph_model* m, int kernel, long long polls);

int mph_model_create(unsigned long long seed, mph_model** out);
void mph_model_destroy(mph_model* m);
int mph_model_param_count(void);
int mph_model_get_params(mph_model* m, float* params);
int mph_model_set_params(mph_model* m, const float* params);
int mph_model_set_scales(mph_model* m, double velocity_scale, double force_scale);
int mph_model_get_scales(mph_model* m, double* velocity_scale, double* force_scale);
/* One forward + backward pass over n host samples: gradient of the mean
 * squared error of the scaled outputs (grad[param_count]) and the loss. */
int mph_model_gradient(mph_model* m, const float* samples, long long n, float* grad, double* loss);
/* Predicted pair forces (N) of n host samples: out[n][4] = (fx, fy, fz, 0). */
int mph_model_predict(mph_model* m, const float* samples, long long n, float* out);
/* Set velocity_scale and force_scale to the RMS of the relative-velocity and
 * target components of the dataset. */
int mph_model_fit_scales(mph_model* m, mph_dataset* d);
/* Adam on shuffled mini-batches of `batch` samples for `epochs` passes over
 * the dataset; *loss gets the mean loss of the last epoch. */
int mph_model_train(mph_model* m, mph_dataset* d, int epochs, int batch, double lr, unsigned long long seed,
                    double* loss);
int mph_model_last_error(mph_model* m, char* buf, int len);

int mph_dataset_create(long long capacity, mph_dataset** out);
void mph_dataset_destroy(mph_dataset* d);
long long mph_dataset_size(mph_dataset* d);
int mph_dataset_append(mph_dataset* d, const float* samples, long long n);
int mph_dataset_read(mph_dataset* d, long long first, long long n, float* samples);
/* Append up to max_samples edges of ctx's current state (fluid particle i,
 * neighbour j within the viscosity radius), drawn at random with the seed,
 * with their FP64 viscous + surface-tension pair force as target.  ctx must
 * be an MPH_MODE_FP64 or MPH_MODE_LEARNED context. */
int mph_collect_samples(mph_ctx* ctx, mph_dataset* d, long long max_samples, unsigned long long seed);

/* Attach a model to an MPH_MODE_LEARNED context (the context keeps a
 * reference; the model must outlive it) with the judge interval and the
 * tolerance of the fallback.  The judged error is the relative L2 error, over
 * the fluid, of the terms the network replaces (PressureA + DiffuseInterface +
 * ViscosityV, main.cpp:1742-1829, 1941-1985) against their FP64 values; when
 * those terms are below 1e-6 of the total force, it is the relative L2 error
 * of the total fluid force instead. */
int mph_set_learned(mph_ctx* ctx, mph_model* m, int judge_interval, double tolerance);
typedef struct mph_learned_info {
    long long steps;           /* steps taken in MPH_MODE_LEARNED              */
    long long learned_steps;   /* steps that used the surrogate                */
    long long judged;          /* judgements (plain step run beside)           */
    long long fallbacks;       /* judgements over the tolerance               */
    long long plain_steps;     /* steps taken by the plain step after a fallback */
    double last_force_error;   /* relative L2 error of the fluid forces        */
    double max_force_error;
    double last_term_error;    /* relative L2 error of the replaced terms (0
                                  when they are below 1e-6 of the total force) */
    double max_term_error;
    long long edges;           /* CSR edges the network evaluates per step     */
    double max_accepted_error; /* largest judged error that was kept (<= tolerance) */
} mph_learned_info;
int mph_learned_stats(mph_ctx* ctx, mph_learned_info* info);

/* ---- batched form: many independent scenes in one step -----------------
 * No counterpart in the reference, which runs one scene per process; each
 * scene here takes the reference's step (main.cpp:386-431, the start-up sort
 * of main.cpp:357-359 included) with the pair arithmetic of
 * MPH_MODE_MIXED_P64 (FP64 density pairs, FP32 force pairs) and FP64
 * integration.  All scenes of a batch have the same dimension; walls
 * must be static (zero Wall2/3 Velocity and Omega).  Scene s keeps its own
 * *.data parameters, domain and cell grid; a step advances every scene by its
 * own dt.  The sweeps are persistent kernels over (scene, cell tile) work
 * items; mph_batch_step replays steps as captured CUDA graphs of
 * MPH_BATCH_GRAPH_STEPS steps (the remainder as direct launches). */
#define MPH_BATCH_GRAPH_STEPS 16
typedef struct mph_batch mph_batch;

/* headers[s].particle_count particles per scene; type, xyz[3], vel[3] hold
 * the scenes' particles one scene after the other, each in its *.grid order. */
int mph_batch_create(int n_scenes, const mph_params* params, const mph_grid_header* headers, int dim,
                     const int* type, const double* xyz, const double* vel, mph_batch** out);
/* Enqueue nsteps steps of every scene on the batch's stream (asynchronous). */
int mph_batch_step(mph_batch* b, int nsteps);
/* Wait for the stream; MPH_ERR_CAPACITY / MPH_ERR_NONFINITE from the device flags. */
int mph_batch_synchronize(mph_batch* b);
/* Positions and velocities of every scene in its input order (layout of
 * mph_batch_create's xyz / vel). */
int mph_batch_get_state(mph_batch* b, double* xyz, double* vel);
/* Cell tile (tz ignored in 2-D), CTA size of the sweeps, and the resident CTAs
 * per SM their staging capacity is sized for (0: keep the current value). */
int mph_batch_set_tiles(mph_batch* b, int tx, int ty, int tz, int threads, int ctas_per_sm);
typedef struct mph_batch_trial {
    int tile[3];
    int threads;
    int ctas_per_sm;   /* resident CTAs per SM the staging capacity is sized for */
    int capacity;      /* particles a CTA stages (tile + halo) before splitting  */
    double ms_per_step;
} mph_batch_trial;
/* Time every candidate tile shape, CTA size and staging capacity (sized for 2
 * to 4 resident CTAs per SM in 2-D, 1 or 2 in 3-D) on the batch itself for about
 * `steps` steps each, keep the fastest, and put the batch state back as it
 * was: the simulation does not advance.  trials[capacity] receives the
 * timings (may be NULL), *count the number of candidates timed. */
int mph_batch_autotune(mph_batch* b, int steps, mph_batch_trial* trials, int capacity, int* count);
typedef struct mph_batch_info {
    int dim, scenes, particles, fluid_particles;
    int tile[3];
    int threads, ctas_per_sm, items, capacity, grid_a, grid_b, graph_steps;
    long long steps;            /* steps taken                                   */
    long long scene_rebuilds;   /* per-scene cell sorts since creation            */
    long long tile_splits;      /* tiles split because their halo did not fit     */
    long long launches;         /* kernels launched                               */
} mph_batch_info;
int mph_batch_get_info(mph_batch* b, mph_batch_info* info);
void* mph_batch_stream(mph_batch* b);
/* Per-kernel-group CUDA-event timing of subsequent steps (direct launches
 * instead of graphs while enabled); read as for mph_profile_read. */
int mph_batch_profile_enable(mph_batch* b, int enable);
int mph_batch_profile_read(mph_batch* b, mph_kernel_stat* out, int capacity, int* count);
int mph_batch_last_error(mph_batch* b, char* buf, int len);
void mph_batch_destroy(mph_batch* b);

/* Last error message of ctx (or of the calling thread if ctx is NULL). */
int mph_last_error(mph_ctx* ctx, char* buf, int len);

void mph_destroy(mph_ctx* ctx);

/* Library version string. */
const char* mph_version(void);

#ifdef __cplusplus
}
#endif

#endif /* MPH_B200_H */
