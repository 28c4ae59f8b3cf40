// mph_io.cpp — the reference's file formats, host side.
//   *.data  : readDataFile     (main.cpp:489-539)
//   *.grid  : readGridFile     (main.cpp:541-640), writeProfFile (672-696)
//   *.vtk   : writeVtkFile     (main.cpp:698-834)
// The sscanf/fprintf patterns are the reference's, so files round-trip
// byte-for-byte between the two programs.  Also the exact binary checkpoint
// (no reference counterpart; see mph_write_checkpoint_arrays).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include "mph_b200.h"
#include "mph_io.h"

extern "C" int mph_params_defaults(mph_params* p) {
    if (!p) return MPH_ERR_ARG;
    std::memset(p, 0, sizeof(*p));
    p->dt = 1.0e100;  // main.cpp:64
    return MPH_OK;
}

extern "C" int mph_read_data_file(const char* path, mph_params* P, int* invalid_lines) {
    if (!path || !P) return MPH_ERR_ARG;
    FILE* fp = std::fopen(path, "r");
    if (!fp) return MPH_ERR_IO;
    char buf[1024];
    int bad = 0;
    double(*W)[3] = P->wall_center;
    double(*U)[3] = P->wall_velocity;
    double(*O)[3] = P->wall_omega;
    double(*IR)[4] = P->interaction_ratio;
    while (!std::feof(fp) && !std::ferror(fp)) {
        if (std::fgets(buf, sizeof(buf), fp) == NULL) continue;
        if (buf[0] == '#') {
        } else if (std::sscanf(buf, " Dt %lf", &P->dt) == 1) {
        } else if (std::sscanf(buf, " OutputInterval %lf", &P->output_interval) == 1) {
        } else if (std::sscanf(buf, " VtkOutputInterval %lf", &P->vtk_output_interval) == 1) {
        } else if (std::sscanf(buf, " EndTime %lf", &P->end_time) == 1) {
        } else if (std::sscanf(buf, " RadiusRatioA %lf", &P->radius_ratio_a) == 1) {
        } else if (std::sscanf(buf, " RadiusRatioP %lf", &P->radius_ratio_p) == 1) {
        } else if (std::sscanf(buf, " RadiusRatioV %lf", &P->radius_ratio_v) == 1) {
        } else if (std::sscanf(buf, " Density %lf %lf %lf %lf", &P->density[0], &P->density[1], &P->density[2],
                               &P->density[3]) == 4) {
        } else if (std::sscanf(buf, " BulkModulus %lf %lf %lf %lf", &P->bulk_modulus[0], &P->bulk_modulus[1],
                               &P->bulk_modulus[2], &P->bulk_modulus[3]) == 4) {
        } else if (std::sscanf(buf, " BulkViscosity %lf %lf %lf %lf", &P->bulk_viscosity[0],
                               &P->bulk_viscosity[1], &P->bulk_viscosity[2], &P->bulk_viscosity[3]) == 4) {
        } else if (std::sscanf(buf, " ShearViscosity %lf %lf %lf %lf", &P->shear_viscosity[0],
                               &P->shear_viscosity[1], &P->shear_viscosity[2], &P->shear_viscosity[3]) == 4) {
        } else if (std::sscanf(buf, " SurfaceTension %lf %lf %lf %lf", &P->surface_tension[0],
                               &P->surface_tension[1], &P->surface_tension[2], &P->surface_tension[3]) == 4) {
        } else if (std::sscanf(buf, " InteractionRatio(Type0) %lf %lf %lf %lf", &IR[0][0], &IR[0][1], &IR[0][2],
                               &IR[0][3]) == 4) {
        } else if (std::sscanf(buf, " InteractionRatio(Type1) %lf %lf %lf %lf", &IR[1][0], &IR[1][1], &IR[1][2],
                               &IR[1][3]) == 4) {
        } else if (std::sscanf(buf, " InteractionRatio(Type2) %lf %lf %lf %lf", &IR[2][0], &IR[2][1], &IR[2][2],
                               &IR[2][3]) == 4) {
        } else if (std::sscanf(buf, " InteractionRatio(Type3) %lf %lf %lf %lf", &IR[3][0], &IR[3][1], &IR[3][2],
                               &IR[3][3]) == 4) {
        } else if (std::sscanf(buf, " Gravity %lf %lf %lf", &P->gravity[0], &P->gravity[1], &P->gravity[2]) == 3) {
        } else if (std::sscanf(buf, " Wall2  Center %lf %lf %lf Velocity %lf %lf %lf Omega %lf %lf %lf", &W[2][0],
                               &W[2][1], &W[2][2], &U[2][0], &U[2][1], &U[2][2], &O[2][0], &O[2][1],
                               &O[2][2]) == 9) {
        } else if (std::sscanf(buf, " Wall3  Center %lf %lf %lf Velocity %lf %lf %lf Omega %lf %lf %lf", &W[3][0],
                               &W[3][1], &W[3][2], &U[3][0], &U[3][1], &U[3][2], &O[3][0], &O[3][1],
                               &O[3][2]) == 9) {
        } else {
            ++bad;  // the reference logs "Invalid line in data file" and goes on
        }
    }
    std::fclose(fp);
    if (invalid_lines) *invalid_lines = bad;
    return MPH_OK;
}

static int read_header_lines(FILE* fp, mph_grid_header* h) {
    char buf[1024];
    if (std::fgets(buf, sizeof(buf), fp) == NULL) return MPH_ERR_IO;
    if (std::sscanf(buf, "%lf", &h->time) != 1) return MPH_ERR_IO;
    if (std::fgets(buf, sizeof(buf), fp) == NULL) return MPH_ERR_IO;
    if (std::sscanf(buf, "%d  %lf  %lf %lf %lf  %lf %lf %lf", &h->particle_count, &h->particle_spacing,
                    &h->domain_min[0], &h->domain_max[0], &h->domain_min[1], &h->domain_max[1],
                    &h->domain_min[2], &h->domain_max[2]) != 8)
        return MPH_ERR_IO;
    if (h->particle_count < 0) return MPH_ERR_IO;
    return MPH_OK;
}

extern "C" int mph_read_grid_header(const char* path, mph_grid_header* h) {
    if (!path || !h) return MPH_ERR_ARG;
    FILE* fp = std::fopen(path, "r");
    if (!fp) return MPH_ERR_IO;
    const int st = read_header_lines(fp, h);
    std::fclose(fp);
    return st;
}

extern "C" int mph_read_grid_file(const char* path, mph_grid_header* h, int capacity, int* type, double* xyz,
                                  double* vel) {
    if (!path || !h || !type || !xyz || !vel) return MPH_ERR_ARG;
    FILE* fp = std::fopen(path, "r");
    if (!fp) return MPH_ERR_IO;
    int st = read_header_lines(fp, h);
    if (st == MPH_OK && h->particle_count > capacity) st = MPH_ERR_ARG;
    char buf[1024];
    for (int i = 0; st == MPH_OK && i < h->particle_count; ++i) {
        if (std::fgets(buf, sizeof(buf), fp) == NULL) { st = MPH_ERR_IO; break; }
        double* q = xyz + 3 * (size_t)i;
        double* v = vel + 3 * (size_t)i;
        if (std::sscanf(buf, "%d  %lf %lf %lf  %lf %lf %lf", &type[i], &q[0], &q[1], &q[2], &v[0], &v[1],
                        &v[2]) != 7) {
            st = MPH_ERR_IO;
            break;
        }
    }
    std::fclose(fp);
    return st;
}

extern "C" int mph_write_grid_file(const char* path, const mph_grid_header* h, const int* type, const double* xyz,
                                   const double* vel) {
    if (!path || !h || (h->particle_count > 0 && (!type || !xyz || !vel))) return MPH_ERR_ARG;
    FILE* fp = std::fopen(path, "w");
    if (!fp) return MPH_ERR_IO;
    std::fprintf(fp, "%e\n", h->time);
    std::fprintf(fp, "%d %e %e %e %e %e %e %e\n", h->particle_count, h->particle_spacing, h->domain_min[0],
                 h->domain_max[0], h->domain_min[1], h->domain_max[1], h->domain_min[2], h->domain_max[2]);
    for (int i = 0; i < h->particle_count; ++i) {
        const double* q = xyz + 3 * (size_t)i;
        const double* v = vel + 3 * (size_t)i;
        std::fprintf(fp, "%d %e %e %e  %e %e %e\n", type[i], q[0], q[1], q[2], v[0], v[1], v[2]);
    }
    std::fflush(fp);
    const int bad = std::ferror(fp);
    std::fclose(fp);
    return bad ? MPH_ERR_IO : MPH_OK;
}

// ---- exact binary checkpoint ---------------------------------------------------
// Layout (native byte order, the struct layouts of mph_b200.h):
//   char magic[8] = "MPHCKPT1"; int32 dim; int32 n; int64 step;
//   mph_params; mph_grid_header; int32 type[n]; int32 particle_index[n];
//   double xyz[3n]; double vel[3n]
namespace {
const char kCkptMagic[8] = {'M', 'P', 'H', 'C', 'K', 'P', 'T', '1'};

struct CkptHead {
    char magic[8];
    int dim, n;
    long long step;
};

int read_ckpt_head(FILE* fp, CkptHead* hd, mph_params* p, mph_grid_header* h) {
    if (std::fread(hd, sizeof(*hd), 1, fp) != 1 || std::memcmp(hd->magic, kCkptMagic, 8) != 0) return MPH_ERR_IO;
    if (std::fread(p, sizeof(*p), 1, fp) != 1 || std::fread(h, sizeof(*h), 1, fp) != 1) return MPH_ERR_IO;
    if ((hd->dim != 2 && hd->dim != 3) || hd->n < 0 || hd->n != h->particle_count) return MPH_ERR_IO;
    return MPH_OK;
}
}  // namespace

extern "C" int mph_write_checkpoint_arrays(const char* path, const mph_params* p, const mph_grid_header* h, int dim,
                                           long long step, const int* type, const int* particle_index,
                                           const double* xyz, const double* vel) {
    if (!path || !p || !h || (dim != 2 && dim != 3) || h->particle_count < 0 ||
        (h->particle_count > 0 && (!type || !particle_index || !xyz || !vel)))
        return MPH_ERR_ARG;
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return MPH_ERR_IO;
    CkptHead hd{};
    std::memcpy(hd.magic, kCkptMagic, 8);
    hd.dim = dim;
    hd.n = h->particle_count;
    hd.step = step;
    const size_t n = (size_t)h->particle_count;
    bool ok = std::fwrite(&hd, sizeof(hd), 1, fp) == 1 && std::fwrite(p, sizeof(*p), 1, fp) == 1 &&
              std::fwrite(h, sizeof(*h), 1, fp) == 1;
    if (ok && n > 0)
        ok = std::fwrite(type, sizeof(int), n, fp) == n && std::fwrite(particle_index, sizeof(int), n, fp) == n &&
             std::fwrite(xyz, sizeof(double), 3 * n, fp) == 3 * n &&
             std::fwrite(vel, sizeof(double), 3 * n, fp) == 3 * n;
    ok = std::fflush(fp) == 0 && ok;
    std::fclose(fp);
    return ok ? MPH_OK : MPH_ERR_IO;
}

extern "C" int mph_read_checkpoint_header(const char* path, mph_params* p, mph_grid_header* h, int* dim,
                                          long long* step) {
    if (!path || !p || !h) return MPH_ERR_ARG;
    FILE* fp = std::fopen(path, "rb");
    if (!fp) return MPH_ERR_IO;
    CkptHead hd{};
    const int st = read_ckpt_head(fp, &hd, p, h);
    std::fclose(fp);
    if (st != MPH_OK) return st;
    if (dim) *dim = hd.dim;
    if (step) *step = hd.step;
    return MPH_OK;
}

extern "C" int mph_read_checkpoint(const char* path, mph_params* p, mph_grid_header* h, int* dim, long long* step,
                                   int capacity, int* type, int* particle_index, double* xyz, double* vel) {
    if (!path || !p || !h || !type || !particle_index || !xyz || !vel) return MPH_ERR_ARG;
    FILE* fp = std::fopen(path, "rb");
    if (!fp) return MPH_ERR_IO;
    CkptHead hd{};
    int st = read_ckpt_head(fp, &hd, p, h);
    if (st == MPH_OK && hd.n > capacity) st = MPH_ERR_ARG;
    const size_t n = (size_t)hd.n;
    if (st == MPH_OK && n > 0 &&
        (std::fread(type, sizeof(int), n, fp) != n || std::fread(particle_index, sizeof(int), n, fp) != n ||
         std::fread(xyz, sizeof(double), 3 * n, fp) != 3 * n || std::fread(vel, sizeof(double), 3 * n, fp) != 3 * n))
        st = MPH_ERR_IO;  // truncated
    std::fclose(fp);
    if (st != MPH_OK) return st;
    if (dim) *dim = hd.dim;
    if (step) *step = hd.step;
    return MPH_OK;
}

namespace mph {

int write_vtk_host(const char* path, int n, const int* type, const double* xyz, const double* vel,
                   const double* force, const int* ncount, const double* dens_a, const double* strain_p,
                   const double* virial_p) {
    FILE* fp = std::fopen(path, "w");
    if (!fp) return MPH_ERR_IO;
    // a large stdio buffer: the file is written sequentially in one pass
    std::vector<char> iobuf(1 << 22);
    std::setvbuf(fp, iobuf.data(), _IOFBF, iobuf.size());
    std::fprintf(fp, "# vtk DataFile Version 2.0\n");
    std::fprintf(fp, "Unstructured Grid Example\n");
    std::fprintf(fp, "ASCII\n");
    std::fprintf(fp, "DATASET UNSTRUCTURED_GRID\n");
    std::fprintf(fp, "POINTS %d float\n", n);
    for (int i = 0; i < n; ++i)
        std::fprintf(fp, "%e %e %e\n", (float)xyz[3 * i], (float)xyz[3 * i + 1], (float)xyz[3 * i + 2]);
    std::fprintf(fp, "CELLS %d %d\n", n, 2 * n);
    for (int i = 0; i < n; ++i) std::fprintf(fp, "1 %d ", i);
    std::fprintf(fp, "\n");
    std::fprintf(fp, "CELL_TYPES %d\n", n);
    for (int i = 0; i < n; ++i) std::fprintf(fp, "1 ");
    std::fprintf(fp, "\n");
    std::fprintf(fp, "\n");
    std::fprintf(fp, "POINT_DATA %d\n", n);
    std::fprintf(fp, "SCALARS label float 1\n");
    std::fprintf(fp, "LOOKUP_TABLE default\n");
    for (int i = 0; i < n; ++i) std::fprintf(fp, "%d\n", type[i]);
    std::fprintf(fp, "\n");
    std::fprintf(fp, "SCALARS DensityA float 1\n");
    std::fprintf(fp, "LOOKUP_TABLE default\n");
    for (int i = 0; i < n; ++i) std::fprintf(fp, "%e\n", (float)dens_a[i]);
    std::fprintf(fp, "\n");
    std::fprintf(fp, "SCALARS VolStrainP float 1\n");
    std::fprintf(fp, "LOOKUP_TABLE default\n");
    for (int i = 0; i < n; ++i) std::fprintf(fp, "%e\n", (float)strain_p[i]);
    std::fprintf(fp, "\n");
    std::fprintf(fp, "SCALARS VirialPressureAtParticle float 1\n");
    std::fprintf(fp, "LOOKUP_TABLE default\n");
    for (int i = 0; i < n; ++i) std::fprintf(fp, "%e\n", (float)virial_p[i]);
    std::fprintf(fp, "\n");
    std::fprintf(fp, "SCALARS neighbor float 1\n");
    std::fprintf(fp, "LOOKUP_TABLE default\n");
    for (int i = 0; i < n; ++i) std::fprintf(fp, "%d\n", ncount[i]);
    std::fprintf(fp, "\n");
    std::fprintf(fp, "VECTORS velocity float\n");
    for (int i = 0; i < n; ++i)
        std::fprintf(fp, "%e %e %e\n", (float)vel[3 * i], (float)vel[3 * i + 1], (float)vel[3 * i + 2]);
    std::fprintf(fp, "\n");
    std::fprintf(fp, "VECTORS force float\n");
    for (int i = 0; i < n; ++i)
        std::fprintf(fp, "%e %e %e\n", (float)force[3 * i], (float)force[3 * i + 1], (float)force[3 * i + 2]);
    std::fprintf(fp, "\n");
    std::fflush(fp);
    const int bad = std::ferror(fp);
    std::fclose(fp);
    return bad ? MPH_ERR_IO : MPH_OK;
}

}  // namespace mph
