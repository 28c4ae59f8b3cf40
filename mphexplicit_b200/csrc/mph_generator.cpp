// mph_generator.cpp — the reference's pre-processor: a *.boid list of cuboids
// turned into a *.grid of particles on each cuboid's lattice
// (generator/generator.cpp of Masahiro-Kondo-AIST/MphExplicit).
//
// The file is read with the same stdio calls and patterns as the reference's
// readfile / readCuboid (generator.cpp:49-164): lines through fgets, '#' lines
// skipped, the first token of a line selects ParticleDistance / LowerDomain /
// UpperDomain / StartCuboid; inside a cuboid, whitespace-separated tokens
// through fscanf up to EndCuboid.  The lattice fill is the reference's loop
// (generator.cpp:170-193): count = round(width / Spacing) (C round, halves
// away from zero), spacing = width / count, coordinates accumulated by
// repeated addition from lower + spacing/2 while below upper - 0.49 spacing,
// in x, y, z nesting order.  The writer prints what the reference's writefile
// prints (generator.cpp:197-217), byte for byte.
//
// Where the reference prints a message and goes on (a missing key, an unknown
// key inside a cuboid) or never returns (a cuboid without EndCuboid), these
// functions return MPH_ERR_IO with the reason instead.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "mph_b200.h"

namespace {

thread_local std::string g_gen_error;

int gen_fail(int code, const std::string& msg) {
    g_gen_error = msg;
    return code;
}

// readCuboid (generator.cpp:111-164): tokens up to `endcommand`.
int read_cuboid(FILE* fp, mph_cuboid* cub) {
    char token[256];
    bool sp = false, ty = false, lo = false, up = false, ve = false;
    std::memset(cub, 0, sizeof(*cub));
    for (;;) {
        const int r = std::fscanf(fp, "%255s", token);
        if (r == EOF) return gen_fail(MPH_ERR_IO, "cuboid without EndCuboid");
        if (r != 1) continue;
        if (std::strcmp(token, "EndCuboid") == 0) break;
        if (std::strcmp(token, "Spacing") == 0) {
            if (std::fscanf(fp, "%lf", &cub->spacing) != 1) return gen_fail(MPH_ERR_IO, "bad Spacing");
            sp = true;
        } else if (std::strcmp(token, "Type") == 0) {
            if (std::fscanf(fp, "%d", &cub->type) != 1) return gen_fail(MPH_ERR_IO, "bad Type");
            ty = true;
        } else if (std::strcmp(token, "Lower") == 0) {
            for (int d = 0; d < 3; ++d)
                if (std::fscanf(fp, "%lf", &cub->lower[d]) != 1) return gen_fail(MPH_ERR_IO, "bad Lower");
            lo = true;
        } else if (std::strcmp(token, "Upper") == 0) {
            for (int d = 0; d < 3; ++d)
                if (std::fscanf(fp, "%lf", &cub->upper[d]) != 1) return gen_fail(MPH_ERR_IO, "bad Upper");
            up = true;
        } else if (std::strcmp(token, "Velocity") == 0) {
            for (int d = 0; d < 3; ++d)
                if (std::fscanf(fp, "%lf", &cub->velocity[d]) != 1) return gen_fail(MPH_ERR_IO, "bad Velocity");
            ve = true;
        } else {
            return gen_fail(MPH_ERR_IO, std::string("unknown cuboid key ") + token);
        }
    }
    if (!(sp && ty && lo && up && ve))
        return gen_fail(MPH_ERR_IO, "a cuboid needs Spacing, Type, Lower, Upper and Velocity");
    return MPH_OK;
}

// Number of lattice points along one axis of a cuboid: the reference's loop
// for (p = lower + 0.5 s; p < upper - 0.49 s; p += s), run as written.
long long axis_points(double lower, double upper, double s, std::vector<double>* out) {
    long long k = 0;
    for (double p = lower + 0.5 * s; p < upper - 0.49 * s; p += s) {
        if (out) out->push_back(p);
        ++k;
    }
    return k;
}

}  // namespace

extern "C" int mph_generator_last_error(char* buf, int len) {
    if (!buf || len <= 0) return MPH_ERR_ARG;
    std::snprintf(buf, (size_t)len, "%s", g_gen_error.c_str());
    return MPH_OK;
}

extern "C" int mph_read_boid_file(const char* path, mph_boid* boid, mph_cuboid* cuboids, int capacity, int* count) {
    if (!path || !boid || !count || capacity < 0 || (capacity > 0 && !cuboids))
        return gen_fail(MPH_ERR_ARG, "bad arguments");
    FILE* fp = std::fopen(path, "r");
    if (!fp) return gen_fail(MPH_ERR_IO, std::string("cannot open ") + path);
    std::memset(boid, 0, sizeof(*boid));
    boid->particle_distance = -1.0;  // generator.cpp:9
    bool pd = false, lo = false, up = false;
    int n = 0;
    int rc = MPH_OK;
    char buf[1024];
    char token[256];
    while (!std::feof(fp) && !std::ferror(fp)) {
        if (std::fgets(buf, sizeof(buf), fp) == nullptr) continue;
        if (buf[0] == '#') continue;
        if (std::sscanf(buf, "%255s", token) != 1) continue;
        if (std::strcmp(token, "ParticleDistance") == 0) {
            if (std::sscanf(buf, " %*s %lf", &boid->particle_distance) != 1) {
                rc = gen_fail(MPH_ERR_IO, "bad ParticleDistance");
                break;
            }
            pd = true;
        } else if (std::strcmp(token, "LowerDomain") == 0) {
            if (std::sscanf(buf, " %*s %lf %lf %lf", &boid->lower_domain[0], &boid->lower_domain[1],
                            &boid->lower_domain[2]) != 3) {
                rc = gen_fail(MPH_ERR_IO, "bad LowerDomain");
                break;
            }
            lo = true;
        } else if (std::strcmp(token, "UpperDomain") == 0) {
            if (std::sscanf(buf, " %*s %lf %lf %lf", &boid->upper_domain[0], &boid->upper_domain[1],
                            &boid->upper_domain[2]) != 3) {
                rc = gen_fail(MPH_ERR_IO, "bad UpperDomain");
                break;
            }
            up = true;
        } else if (std::strcmp(token, "StartCuboid") == 0) {
            mph_cuboid c;
            rc = read_cuboid(fp, &c);
            if (rc != MPH_OK) break;
            if (n < capacity) cuboids[n] = c;
            ++n;
        }
    }
    std::fclose(fp);
    if (rc != MPH_OK) return rc;
    if (!(pd && lo && up)) return gen_fail(MPH_ERR_IO, "a *.boid file needs ParticleDistance, LowerDomain and UpperDomain");
    boid->cuboid_count = n;
    *count = n;
    if (n > capacity) return gen_fail(MPH_ERR_CAPACITY, "more cuboids than the capacity");
    return MPH_OK;
}

extern "C" int mph_generate_cuboids(const mph_cuboid* cuboids, int count, int* type, double* xyz, double* vel,
                                    long long capacity, long long* n) {
    if (count < 0 || (count > 0 && !cuboids) || !n || capacity < 0) return gen_fail(MPH_ERR_ARG, "bad arguments");
    const bool fill = type && xyz && vel;
    long long k = 0;
    std::vector<double> ax[3];
    for (int c = 0; c < count; ++c) {
        const mph_cuboid& cub = cuboids[c];
        double width[3], s[3];
        int cnt[3];
        for (int d = 0; d < 3; ++d) {
            width[d] = cub.upper[d] - cub.lower[d];
            cnt[d] = (int)std::round(width[d] / cub.spacing);  // generator.cpp:175
            s[d] = width[d] / cnt[d];                            // generator.cpp:176
        }
        // the loop bounds depend only on their own axis, so the nest is the
        // outer product of the three axis sequences, in x, y, z order
        for (int d = 0; d < 3; ++d) {
            ax[d].clear();
            axis_points(cub.lower[d], cub.upper[d], s[d], &ax[d]);
        }
        for (double px : ax[0])
            for (double py : ax[1])
                for (double pz : ax[2]) {
                    if (fill) {
                        if (k >= capacity) return gen_fail(MPH_ERR_CAPACITY, "more particles than the capacity");
                        type[k] = cub.type;
                        xyz[3 * k] = px;
                        xyz[3 * k + 1] = py;
                        xyz[3 * k + 2] = pz;
                        for (int d = 0; d < 3; ++d) vel[3 * k + d] = cub.velocity[d];
                    }
                    ++k;
                }
    }
    *n = k;
    return MPH_OK;
}

extern "C" int mph_write_generated_grid(const char* path, const mph_boid* boid, long long n, const int* type,
                                        const double* xyz, const double* vel) {
    if (!path || !boid || n < 0 || (n > 0 && (!type || !xyz || !vel))) return gen_fail(MPH_ERR_ARG, "bad arguments");
    if (n > 0x7fffffffLL) return gen_fail(MPH_ERR_CAPACITY, "particle count does not fit the file's int");
    FILE* fp = std::fopen(path, "w");
    if (!fp) return gen_fail(MPH_ERR_IO, std::string("cannot write ") + path);
    std::fprintf(fp, "%lf\n", 0.0);
    std::fprintf(fp, "%d %e  %e %e %e  %e %e %e\n", (int)n, boid->particle_distance, boid->lower_domain[0],
                 boid->upper_domain[0], boid->lower_domain[1], boid->upper_domain[1], boid->lower_domain[2],
                 boid->upper_domain[2]);
    for (long long i = 0; i < n; ++i)
        std::fprintf(fp, "%d   %e %e %e    %e %e %e\n", type[i], xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2],
                     vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
    std::fflush(fp);
    const int bad = std::ferror(fp);
    std::fclose(fp);
    return bad ? gen_fail(MPH_ERR_IO, std::string("write failed: ") + path) : MPH_OK;
}

extern "C" int mph_generate_grid_file(const char* boid_path, const char* grid_path, long long* particle_count) {
    if (!boid_path || !grid_path) return gen_fail(MPH_ERR_ARG, "bad arguments");
    mph_boid boid;
    int count = 0;
    int rc = mph_read_boid_file(boid_path, &boid, nullptr, 0, &count);
    if (rc != MPH_OK && rc != MPH_ERR_CAPACITY) return rc;
    std::vector<mph_cuboid> cub((size_t)count);
    rc = mph_read_boid_file(boid_path, &boid, cub.data(), count, &count);
    if (rc != MPH_OK) return rc;
    long long n = 0;
    rc = mph_generate_cuboids(cub.data(), count, nullptr, nullptr, nullptr, 0, &n);
    if (rc != MPH_OK) return rc;
    std::vector<int> type((size_t)n);
    std::vector<double> xyz(3 * (size_t)n), vel(3 * (size_t)n);
    rc = mph_generate_cuboids(cub.data(), count, type.data(), xyz.data(), vel.data(), n, &n);
    if (rc != MPH_OK) return rc;
    rc = mph_write_generated_grid(grid_path, &boid, n, type.data(), xyz.data(), vel.data());
    if (rc == MPH_OK && particle_count) *particle_count = n;
    return rc;
}
